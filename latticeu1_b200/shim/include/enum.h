// Enumerations of the reference's API (reference include/enum.h:13-31).
#ifndef U1_SHIM_ENUM_H
#define U1_SHIM_ENUM_H
namespace U1 {
typedef enum Verbosity_s { SILENT, SUMMARIZE, VERBOSE, DEBUG_VERBOSE } Verbosity;
typedef enum TuneMode_S { TUNE_NO, TUNE_YES } TuneMode;
typedef enum ReadMode_S { Host, Device } ReadMode;
}  // namespace U1
#endif
