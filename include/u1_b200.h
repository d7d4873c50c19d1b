/*
 * u1_b200.h -- C ABI of the B200 (sm_100a) U(1) lattice-gauge Monte Carlo hot path.
 *
 * Every entry point returns an int status (U1_OK == 0).  Handles are opaque,
 * there is no process-global lattice state, nothing calls exit(), and every
 * device operation runs on the stream attached to the lattice (default: the
 * legacy stream 0).  On failure u1_last_error() returns a thread-local message.
 *
 * Link layout at the boundary (import/export): the reference's FP64 angle
 * array theta[id + parity*V/2 + mu*V], id = even/odd site index
 * (reference include/index.h:114-153, u1.cpp:99, src/update.cu:188).
 * Internally a link is a float2 (cos theta, sin theta) stored at the same index.
 *
 * Geometry follows reference src/parameters.cu:146-208: N = {Nx, Ny, Nz, Nt}
 * is given in the reference's argument order and mapped onto Grid[] the way
 * SetupLatticeParameters does (2D: Grid = {Nx, Nt}; 3D: {Nx, Ny, Nt}).
 */
#ifndef U1_B200_H
#define U1_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
  U1_OK = 0,
  U1_ERR_INVALID = -1,     /* bad argument (odd extent, null pointer, ...) */
  U1_ERR_CUDA = -2,        /* a CUDA runtime call failed */
  U1_ERR_UNSUPPORTED = -3, /* valid request outside what this build supports */
  U1_ERR_NOMEM = -4,       /* device or host allocation failed */
  U1_ERR_STATE = -5        /* object in the wrong state (e.g. replay stream exhausted) */
};

typedef struct u1_ctx u1_ctx;
typedef struct u1_lattice u1_lattice;
typedef struct u1_rng u1_rng;
typedef struct u1_batch u1_batch;

typedef struct u1_geom {
  int dims;       /* 2, 3 or 4 (reference "dirs") */
  int N[4];       /* Nx, Ny, Nz, Nt in the reference's argument order; unused entries ignored */
  double beta;    /* reference "beta" */
  double aniso;   /* reference "aniso" (xi): spatial plaquettes weighted 1/xi, temporal xi */
} u1_geom;

/* Last error message of the calling thread ("" if none). */
const char *u1_last_error(void);
/* Library version string. */
const char *u1_version(void);

/* Device allocator of the whole library.  Replaces the allocation layer of the
 * reference's dev_malloc_ / dev_free_ (reference src/alloc.cpp:178-200,
 * 321-340), which always call cudaMalloc / cudaFree and exit() on failure.
 * alloc(user, bytes, &ptr) returns 0 and a device pointer, or nonzero on
 * failure (the library then returns U1_ERR_NOMEM and the object it was
 * working on stays usable); release(user, ptr) returns a block, and is called
 * only after the device has finished all work (the library synchronises the
 * device first, as cudaFree does).  Give both or
 * neither (NULL, NULL restores cudaMalloc / cudaFree).  Lets a host framework
 * place the library's memory in its own pool, and lets tests inject
 * allocation failures on the host.  Refused with U1_ERR_STATE while the
 * library holds blocks from the current allocator (destroy every object
 * first).  Not for concurrent use with other calls of this library. */
typedef int (*u1_dev_alloc_fn)(void *user, size_t bytes, void **out);
typedef void (*u1_dev_free_fn)(void *user, void *ptr);
int u1_set_device_allocator(u1_dev_alloc_fn alloc, u1_dev_free_fn release, void *user);
/* Device blocks the library currently holds (all allocators; leak checks). */
int u1_device_allocations(int64_t *live);

/* Replaces Start(gpuid, ...) (reference src/cuda_error_check.cpp:24-45):
 * selects the device; no tune-cache side effects. */
int u1_ctx_create(int device, u1_ctx **out);
/* Replaces Finalize (reference src/cuda_error_check.cpp:47-72) without exit(). */
int u1_ctx_destroy(u1_ctx *ctx);
/* Stream used by lattices created after this call (cudaStream_t as void*). */
int u1_ctx_set_stream(u1_ctx *ctx, void *stream);

/* Host-only geometry check and sizes, no device needed (reference
 * SetupLatticeParameters' Grid/volume logic, src/parameters.cu:150-166):
 * out[0]=V, out[1]=V/2, out[2]=V_s, out[3]=dims, out[4..7]=Grid[0..3].
 * Odd or non-positive extents return U1_ERR_INVALID. */
int u1_geom_validate(const u1_geom *geom, int64_t out[8]);

/* Replaces SetupLatticeParameters (reference src/parameters.cu:146-208) plus
 * new Array<double>(Device, Volume()*Dirs()) (reference u1.cpp:99): allocates
 * a cold (theta = 0) lattice, as the reference's zero-filled dev_malloc does
 * (reference src/alloc.cpp:193).  Odd extents return U1_ERR_INVALID
 * (reference src/parameters.cu:164-168 exits instead). */
int u1_lattice_create(u1_ctx *ctx, const u1_geom *geom, u1_lattice **out);
int u1_lattice_destroy(u1_lattice *lat);
/* Attach a stream (cudaStream_t as void*; NULL = legacy default stream). */
int u1_lattice_set_stream(u1_lattice *lat, void *stream);
/* Sizes: out[0]=V, out[1]=V/2, out[2]=V_s, out[3]=dims, out[4..7]=Grid[0..3]. */
int u1_lattice_info(const u1_lattice *lat, int64_t out[8]);
/* Change beta / aniso of an existing lattice (no reallocation). */
int u1_lattice_set_coupling(u1_lattice *lat, double beta, double aniso);
/* Sweeps issued by u1_update are captured once into a CUDA graph and
 * replayed (enable = 1, default) or launched kernel by kernel (enable = 0).
 * Both issue the same kernels with the same arguments. */
int u1_lattice_set_graphs(u1_lattice *lat, int enable);
/* Update kernel variants, all giving bit-identical links: 1 = two sites per
 * thread (32-register cap, 8 CTAs/SM), 2 = two sites per thread (no cap),
 * 3 = one site per thread, 5 = four sites per thread (72-register cap,
 * 256-bit loads, at most 128 threads per block: larger settings run 128); 0 = auto (tuned at the first u1_update among 1, 2, 3, 5).
 * The two-site variants need Nx/2 even, the four-site one Nx/2 a multiple
 * of 4.  4 = the whole sweep as one
 * persistent cooperative kernel with neighbour-local phase synchronisation
 * (4D, (Nx/2)*Ny/2 a multiple of 32 in [64, 256], every (z, t) tile resident
 * at once; opt-in, slower than 1 on B200 at 32^4). */
int u1_lattice_set_variant(u1_lattice *lat, int variant);
/* The variant in use: 0 while automatic and not yet tuned. */
int u1_lattice_get_variant(const u1_lattice *lat, int *variant);
/* Waits of the persistent sweep (variant 4; no counterpart in the reference):
 * each neighbour wait polls at most spin_limit times (0: the default, about a
 * second), and stall_tile >= 0 names a tile that never publishes its phases,
 * a test hook whose neighbours' waits then run out.  A wait that runs out ends
 * the sweep early and leaves the configuration invalid; the next synchronous
 * call on the lattice returns U1_ERR_CUDA and clears the condition. */
int u1_lattice_set_wave_wait(u1_lattice *lat, unsigned spin_limit, int stall_tile);
/* Metropolis proposal (no reference counterpart; the reference proposes
 * theta' = 2 pi u on the whole circle, once per link and pass,
 * src/update.cu:181-182, and that stays the default: delta = 0, nhits = 1).
 * nhits (1..127) hits per link and Metropolis pass, the staple held fixed;
 * hit h proposes theta' = theta + delta (2u - 1) for delta in (0, pi]
 * (theta' = 2 pi u for delta = 0) and accepts when
 * exp(beta Re(S (U' - U))) > b.  Hit h draws its (u, b) from the Philox
 * counter of the pass with stream tag 0 for h = 0 and 0x80 | h for h >= 1.
 * Applies to u1_update, u1_update_measure, u1_update_phase and the
 * multilevel sub-updates of this lattice; the persistent variant 4 is then
 * replaced by the default phase kernels. */
int u1_lattice_set_metropolis(u1_lattice *lat, double delta, int nhits);
int u1_lattice_get_metropolis(const u1_lattice *lat, double *delta, int *nhits);
/* Replaces the reference's autotuner (tuneLaunch, src/tune.cpp:306-416):
 * times every valid variant (1, 2, 3, 5) at 64, 96, 128, 192 and 256 threads per block (5: up to 128) on a
 * few sweeps of this lattice from a backed-up state (links and rng pass
 * restored afterwards), keeps the fastest pair and caches it per (device,
 * geometry); with U1_RESOURCE_PATH set the cache persists in
 * $U1_RESOURCE_PATH/u1b200_tunecache.tsv.  U1_TUNE=0 in the environment
 * turns the automatic first-update tuning off.  *variant gets the variant;
 * u1_lattice_get_block the block size. */
int u1_tune(u1_lattice *lat, u1_rng *rng, int *variant);
/* Threads per block of the phase kernels of variants 1, 2, 3, 5 (32, ..., 256;
 * default 256; the reference's block.x, include/tune.h:143-260).  Every block
 * size gives bit-identical links.  The measuring phases of a measured sweep
 * and the persistent variant keep their own block sizes. */
int u1_lattice_set_block(u1_lattice *lat, int threads);
int u1_lattice_get_block(const u1_lattice *lat, int *threads);
/* Device pointer of the float2 link array (V*dims float2). */
int u1_lattice_links(u1_lattice *lat, void **dev_ptr);
/* Copy all links of src into dst (same geometry). */
int u1_lattice_copy(u1_lattice *dst, const u1_lattice *src);

/* Import/export in the reference layout theta[id + p*V/2 + mu*V] (FP64).
 * on_device != 0: the pointer is a device pointer on the lattice's device. */
int u1_lattice_import_angles(u1_lattice *lat, const double *angles, int on_device);
int u1_lattice_export_angles(const u1_lattice *lat, double *angles, int on_device);
/* Asynchronous forms (no counterpart in the reference, whose Array<double>
 * stays on the device): queued on the lattice's stream behind the work
 * already there, they return at once.  A host buffer should be page-locked
 * (cudaHostAlloc / cudaHostRegister) and left alone until the stream has
 * passed the copy; a pageable one still works, but then the copy blocks the
 * host.  Lattices on separate streams so overlap one lattice's host-to-device
 * copy with another's device-to-host copy and sweeps.  A failed wait of the
 * persistent variant 4 is reported by the next synchronous call. */
int u1_lattice_import_angles_async(u1_lattice *lat, const double *angles, int on_device);
int u1_lattice_export_angles_async(const u1_lattice *lat, double *angles, int on_device);
/* Wait for everything queued on the lattice's stream. */
int u1_lattice_synchronize(u1_lattice *lat);
/* Cold start: every theta = 0. */
int u1_cold_start(u1_lattice *lat);

/* Counter-based RNG (Philox4x32-10).  Replaces CudaRNG(seed, V/2)
 * (reference include/random.h:31-58, src/random.cu:28-36): the state is
 * (seed, pass counter) only, so it is free to checkpoint and any thread or
 * tile order draws the same numbers. */
int u1_rng_create(u1_ctx *ctx, uint64_t seed, u1_rng **out);
int u1_rng_destroy(u1_rng *rng);
int u1_rng_get_state(const u1_rng *rng, uint64_t *seed, uint64_t *pass);
int u1_rng_set_state(u1_rng *rng, uint64_t seed, uint64_t pass);
/* Chain number (0..65535) folded into every Philox counter: independent
 * chains (one per GPU, or per lattice of a batch) share a seed and still
 * draw disjoint streams. */
int u1_rng_set_chain(u1_rng *rng, uint32_t chain);
/* Test-only shared-stream mode: Metropolis passes read (new_theta, b) pairs
 * from `pairs` (host FP64, 2 values per link) in the reference's draw order
 * pass -> parity -> mu -> id (reference src/update.cu:51-79, 305-308).
 * n_pairs must be a multiple of V*dims (one pass).  NULL/0 switches back
 * to Philox. */
int u1_rng_set_replay(u1_rng *rng, const double *pairs, size_t n_pairs);
/* The uniforms Philox gives link (parity, mu, id) in Metropolis pass `pass`
 * for the lattice's geometry: out[2*id], out[2*id+1] (float, as drawn). */
int u1_rng_debug_uniforms(u1_lattice *lat, const u1_rng *rng, uint64_t pass,
                          int parity, int mu, float *out_host);

/* Replaces HotStart (reference src/update.cu:30-48): theta uniform in
 * [0, 2 pi) for every link, drawn from the rng (tag "hot start"). */
int u1_hot_start(u1_lattice *lat, u1_rng *rng);

/* Replaces UpdateLattice (reference src/update.cu:449-456): metrop
 * Metropolis passes, then ovrn overrelaxation passes; each pass visits
 * parity 0,1 and mu = 0..dims-1 in order (reference src/update.cu:305-308,
 * 383-386).  Asynchronous on the lattice's stream. */
int u1_update(u1_lattice *lat, u1_rng *rng, int metrop, int ovrn);

/* u1_update followed by the plaquette + Polyakov measurement of the new
 * configuration (the reference driver's UpdateLattice then Plaquette and
 * Polyakov, u1.cpp:120-126), with the plaquettes taken from the staples of
 * the sweep's last pass and one Polyakov kernel after it: dev_out (device,
 * 6 doubles) receives {SS re, SS im, ST re, ST im, L re, L im} as
 * u1_measure.  The links are bit-identical to u1_update.  Asynchronous. */
int u1_update_measure(u1_lattice *lat, u1_rng *rng, int metrop, int ovrn, double *dev_out);

/* Test and debugging aid: run exactly one (parity, mu) phase of a
 * Metropolis (metropolis != 0) or overrelaxation pass, with the Metropolis
 * numbers of pass (rng pass counter + hit).  The pass counter is not
 * advanced.  A pass of u1_update is the phases parity 0,1 x mu 0..dims-1 in
 * that order (reference src/update.cu:305-308). */
int u1_update_phase(u1_lattice *lat, u1_rng *rng, int metropolis, int parity, int mu, int hit);

/* Replaces Plaquette (reference src/plaquette.cu:222-228):
 * out = {SS re, SS im, ST re, ST im} of mean(1 - exp(i theta_P)).  In 2D the
 * SS mean has no plaquettes and is NaN, as in the reference. Synchronous. */
int u1_plaquette(u1_lattice *lat, double out[4]);
/* Replaces Polyakov (reference src/polyakov.cu:169-174): out = {re, im} of
 * (1/V_s) sum_x exp(i sum_t theta_t(x,t)).  Synchronous. */
int u1_polyakov(u1_lattice *lat, double out[2]);
/* Fused plaquette + Polyakov pass: out = {SS re, SS im, ST re, ST im, L re, L im}. */
int u1_measure(u1_lattice *lat, double out[6]);
/* Asynchronous form: the 6 doubles land in device memory dev_out. */
int u1_measure_async(u1_lattice *lat, double *dev_out);

/* No counterpart in the reference.  The u1_measure_async measurement for
 * callers that cannot allocate device memory (e.g. code confined to memory
 * handed out by its host framework, or loops where a cudaMalloc that may
 * synchronise the device is not acceptable).  It allocates nothing: its
 * scratch is a fixed file-scope device array of about 384 KiB that every GPU
 * loading the library keeps until exit.  links_dev: the V*dims float2 links
 * (this library's layout); out_dev: 6 doubles, as u1_measure; stream:
 * cudaStream_t as void* on the current device.  Lattices with V/2 above
 * 1,048,576 sites return U1_ERR_INVALID.  The first call on a device (and
 * the first after the device's CUDA context changes, e.g. cudaDeviceReset)
 * looks up the array's address and should come before any stream capture;
 * calls that overlap on the GPU race on the shared array. */
int u1_measure_noalloc(const void *links_dev, const u1_geom *geom, double *out_dev, void *stream);

/* Replaces Poly2 (reference src/polyakov.cu:618-654):
 * out[2*(r-1)], out[2*(r-1)+1] = re, im of C(r) for r = 1..R, R = Grid[0]/2,
 * C(r) = 1/(V_s (d-1)) sum_x sum_i P(x) conj(P(x + r e_i)).  multihit != 0
 * replaces each temporal link by its analytic multihit mean
 * (reference include/lattice_functions.h:92-105). */
int u1_poly_corr(u1_lattice *lat, int multihit, double *out, int out_len);

/* Replaces MultiLevel (reference src/multilevel.cu:639-732).  Works on an
 * internal copy of the lattice (the caller's links are unchanged) and
 * advances the rng.  Requires dims == 4 and Nt % 4 == 0 (else U1_ERR_INVALID;
 * the reference exits).  out as for u1_poly_corr.  The first call allocates
 * the work buffers (working copy, slab products and the two tensors: about
 * 210 MB at 24^3 x 32) and they stay with the lattice until it is destroyed,
 * as do the graphs of the last (n2-independent) sub-update shape and rng. */
int u1_multilevel(u1_lattice *lat, u1_rng *rng, int n4, int k4, int n2, int k2,
                  int metrop, int ovrn, double *out, int out_len);

/* ------------------------------------------------------------------ batches
 * Many independent chains advanced by shared launches.  The reference runs
 * one lattice per process (u1.cpp:99-120, one UpdateLattice call per
 * sweep); a batch advances nchains lattices (same dims, any extents, own
 * beta and aniso each) with one kernel per (parity, mu) phase for all of
 * them, and captures each sweep shape once as a CUDA graph.  All chains
 * share the Philox key `seed`; chain c uses chain number first_chain + c in
 * the counter, so it follows exactly the trajectory of a single lattice
 * driven by u1_update with an rng of the same seed, u1_rng_set_chain(
 * first_chain + c), and the same sequence of hot starts and updates.
 * first_chain + nchains <= 65536.  Chains start cold. */
int u1_batch_create(u1_ctx *ctx, int nchains, const u1_geom *geoms, uint64_t seed, uint32_t first_chain,
                    u1_batch **out);
int u1_batch_destroy(u1_batch *b);
int u1_batch_set_stream(u1_batch *b, void *stream);
/* out = {nchains, dims, total links, two-sites-per-thread kernels in use}. */
int u1_batch_info(const u1_batch *b, int64_t out[4]);
/* Number of chain groups a sweep runs one after another (consecutive chains
 * whose links fit comfortably in L2, so that each group's sweep after its
 * first phase is served from L2).  The result is the same as one group.
 * The untuned group size is U1_BATCH_GROUP_MB MiB (default 32; 0: one
 * group), read at u1_batch_create. */
int u1_batch_groups(const u1_batch *b, int *groups);
/* Autotuner of the batch (replaces the reference's per-kernel block-size
 * search, src/tune.cpp:306-416, for many chains per launch): the group size
 * (32 ... 96 MiB of links) and the lanes (below), then, per group, the update
 * kernel (four, two or one site per thread) and threads per block, timed as
 * graph-replayed sweeps
 * from a backed-up state (links and pass counter restored).  Every choice
 * gives the same links bit for bit.  Cached per (device, dims, chain
 * extents) in memory and in $U1_RESOURCE_PATH/u1b200_batch_tunecache.tsv;
 * a cached result is applied without trials.  *group_mb (may be NULL) gets
 * the chosen group size in MiB.  Synchronous; not inside a stream capture. */
int u1_batch_tune(u1_batch *b, int *group_mb);
/* Explicit layout (no counterpart in the reference): groups of at most
 * group_mb MiB (<= 0: keep the current size); group k gets kernel
 * variants[k] (5: four sites per thread, 1: two, 3: one) at threads[k]
 * threads per block for k < ngroups; other groups, or choices a group's
 * chains do not allow, take the default (four sites at 128 threads where
 * every chain has Nx/2 a multiple of 4, else two sites at 256 where Nx/2 is
 * even, else one site at 256). */
int u1_batch_configure(u1_batch *b, int group_mb, int ngroups, const int *variants, const int *threads);
/* Group `group`: out = {first chain, end chain, variant, threads per block}. */
int u1_batch_group_info(const u1_batch *b, int group, int out[4]);
/* Lanes of a sweep (no counterpart in the reference): 1 sweeps the groups
 * one after another on the batch's stream; 2 (the default, U1_BATCH_LANES=1
 * at u1_batch_create for one) alternates them between that stream and a
 * second one forked from and joined back into it within the sweep, so one
 * group's phase boundaries overlap another group's phases.  The links are
 * the same either way; the tuner picks the count. */
int u1_batch_set_lanes(u1_batch *b, int lanes);
int u1_batch_get_lanes(const u1_batch *b, int *lanes);
/* Hot start of every chain (as u1_hot_start); advances the pass counter by 1. */
int u1_batch_hot_start(u1_batch *b);
/* One sweep of every chain: metrop Metropolis then ovrn overrelaxation
 * passes (as u1_update).  measure != 0 appends the plaquette + Polyakov
 * measurement of every chain; read it with u1_batch_results.  Asynchronous. */
int u1_batch_update(u1_batch *b, int metrop, int ovrn, int measure);
/* Measure every chain now: out_host = 6 doubles per chain (as u1_measure). */
int u1_batch_measure(u1_batch *b, double *out_host);
/* The last measurement (6 doubles per chain), waiting for the batch's stream. */
int u1_batch_results(u1_batch *b, double *out_host);
/* Device address of the 6*nchains result doubles (valid until destroy). */
int u1_batch_results_device(u1_batch *b, double **dev_ptr);
/* Per-chain FP64 angles in the reference's EO layout (as u1_lattice_*_angles). */
int u1_batch_import_angles(u1_batch *b, int chain, const double *angles_host);
int u1_batch_export_angles(u1_batch *b, int chain, double *angles_host);
/* Every chain's FP64 angles into device memory angles_dev (total-links
 * doubles, chain after chain in creation order, each in the reference's EO
 * layout).  Asynchronous on the batch's stream. */
int u1_batch_export_all(u1_batch *b, double *angles_dev);
/* Metropolis passes done so far (the rng pass counter of the batch). */
int u1_batch_get_pass(const u1_batch *b, uint64_t *pass);

/* ------------------------------------------------------------ Wilson action
 * No counterpart in the reference (which never evaluates the action or its
 * gradient; its per-plaquette angle is the one summed in src/plaquette.cu:
 * 93-118, its staple weights include/staple.h:75-102).  For `batch`
 * configurations theta_dev[b][mu*V + parity*V/2 + eo] (the reference's angle
 * layout; dtype 0 = float, 1 = double; device memory):
 *   S_b = beta sum_x sum_{mu<nu} w_{mu nu} (1 - cos theta_P(x)),
 *   w = 1/aniso (spatial-spatial) or aniso (with the time direction),
 * out_dev[2b] = S_b and out_dev[2b+1] = the topological charge
 * Q_b = (1/2pi) sum_x wrap(theta_P(x)) in 2D (0 otherwise), FP64 sums in a
 * fixed order.  workspace: u1_action_workspace_bytes of device memory.
 * Nothing is allocated; all work is queued on `stream` (cudaStream_t). */
int u1_action_workspace_bytes(const u1_geom *geom, int batch, size_t *bytes);
int u1_wilson_action(const u1_geom *geom, const void *theta_dev, int dtype, int batch, void *workspace,
                     double *out_dev, void *stream);
/* Adjoint: grad_dev[b][link] = scale_dev[b] * dS_b/dtheta(link)
 * = scale * beta sum_{nu != mu} w [sin theta_{mu nu}(x) - sin theta_{mu nu}(x - nu)]
 * (scale_dev may be NULL for 1), same dtype and layout as theta. */
int u1_wilson_action_grad(const u1_geom *geom, const void *theta_dev, int dtype, int batch,
                          const double *scale_dev, void *grad_dev, void *stream);

/* ------------------------------------------------------------------ formats
 * Replaces ConvLattice_EO_NO (reference src/convertOrder.cu:32-63): FP64
 * angle arrays (device memory, V*dims doubles) between the even/odd order
 * theta[eo + parity*V/2 + mu*V] and the natural order theta[lex + mu*V],
 * lex = x0 + N0*(x1 + N1*(x2 + N2*x3)).  eo_to_no != 0: EO -> NO.  in and
 * out must not alias.  Queued on `stream`. */
int u1_convert_order(const u1_geom *geom, const double *in_dev, double *out_dev, int eo_to_no, void *stream);
/* Replaces PlaquetteFields(lat, field, spacetime, evenoddOrder=true)
 * (reference src/plaquette_comps.cu:34-107, :220-235; 4D only): the six
 * components (mu,nu) = (0,3),(1,3),(2,3),(1,2),(2,0),(0,1) of 1 - e^{i theta_P}
 * as complex FP64 (re, im) pairs.  spacetime != 0: field_dev[2*(lex + d*V)],
 * one value per site; else field_dev[2*(lex_s + d*V_s)], the time average at
 * each spatial site (lex_s = x0 + N0*(x1 + N1*x2)).  means = the six
 * component means (re, im) over the field.  Synchronous. */
int u1_plaquette_fields(u1_lattice *lat, int spacetime, double *field_dev, double means[12]);
/* Configuration checkpoints (no counterpart in the reference, which has no
 * configuration I/O).  Version-1 file: a 128-byte header (magic "U1B200CK",
 * geometry, beta, aniso, rng seed, pass and chain, flags, CRC-32s), the FP64
 * angles in the reference's EO layout, and with exact != 0 the float2 links
 * as well, so that u1_checkpoint_load resumes the chain bit for bit (without
 * them the links are rebuilt from the angles).  rng may be NULL (saved as
 * zeros / left unchanged).  Load checks the geometry, the CRCs, sets beta
 * and aniso from the file and the rng's seed, pass and chain. */
int u1_checkpoint_save(u1_lattice *lat, const u1_rng *rng, const char *path, int exact);
int u1_checkpoint_load(u1_lattice *lat, u1_rng *rng, const char *path);
/* Header of a checkpoint (no device work): geometry in this ABI's
 * (Nx, Ny, Nz, Nt) convention, rng state and flags (bit 0: exact links). */
int u1_checkpoint_info(const char *path, u1_geom *geom, uint64_t *seed, uint64_t *pass, uint32_t *chain,
                       uint32_t *flags);

/* --------------------------------------------------------- flow transform
 * No counterpart in the reference.  Elementwise circular coupling transform
 * of the 2D gauge-equivariant flow (mixture of K <= 8 non-compact
 * projections on plaquette angles, after Kanwar et al., arXiv:2003.06413).
 * n elements, FP32 device buffers; params[e*(2K+1) + .] = (a_0..a_{K-1},
 * logit_0..logit_{K-1}, shift), alpha_k = exp(a_k) (a clamped to [-8, 8]),
 * w = softmax(logit).  With xc = remainder(x, 2 pi) and
 * H(xc) = sum_k w_k 2 atan2(alpha_k sin(xc/2), cos(xc/2)):
 *   forward:  dy = H(xc) + shift - xc,  logd = log H'(xc)
 *   inverse:  z = remainder(y - shift, 2 pi), xsol solves H(xsol) = z,
 *             dx = xsol - z - shift,  logd = log H'(xsol)
 * The backward entry points take the upstream gradients (either may be NULL
 * for zero) and write the input and parameter gradients.  Queued on `stream`. */
int u1_ncp_forward(const float *x, const float *params, int64_t n, int K, float *dy, float *logd, void *stream);
int u1_ncp_backward(const float *x, const float *params, const float *gdy, const float *glogd, int64_t n, int K,
                    float *gx, float *gparams, void *stream);
int u1_ncp_inverse(const float *y, const float *params, int64_t n, int K, float *dx, float *xsol, float *logd,
                   void *stream);
int u1_ncp_inverse_backward(const float *xsol, const float *params, const float *gdx, const float *glogd, int64_t n,
                            int K, float *gy, float *gparams, void *stream);

/* One whole coupling layer of the 2D flow, forward only (no counterpart in
 * the reference): batch configurations theta_in[b][mu][x1][x0] (L x L,
 * float32, device) -> theta_out, logdet[b] = sum of log H' over the layer's
 * active plaquettes.  Layer (mu, off): links of direction mu on stripes
 * x_nu = off (mod 4) change through their + plaquette; the context net sees
 * (cos P, sin P) of the frozen plaquettes ((x_nu - off) mod 4 in {1, 2}):
 * conv3x3(2 -> hidden; W1, B1), LeakyReLU(slope), conv3x3(hidden -> 2K+1;
 * W2, B2), circular padding, weights rounded to bfloat16, FP32 arithmetic.
 * L a multiple of 4 up to 32, K <= 8, hidden a multiple of 4 up to 32.  Queued on
 * `stream`. */
int u1_flow_layer_forward(const float *theta_in, float *theta_out, float *logdet, int batch, int L, int mu, int off,
                          int K, int hidden, const float *W1, const float *B1, const float *W2, const float *B2,
                          float slope, void *stream);

/* Backward of u1_flow_layer_forward (L up to 32): from theta_in and the
 * upstream gradients grad_theta_out (batch x 2 x L x L) and grad_logdet
 * (batch; NULL for zero), writes grad_theta_in and the weight gradients
 * wgrad = (dW1[c][ci][ky][kx], dB1[c], dW2[o][ci][ky][kx], dB2[o]) summed over
 * the batch in a fixed order (with respect to the bf16-rounded weights the
 * forward uses).  wgrad_partials: batch * len(wgrad) floats of scratch. */
int u1_flow_layer_backward(const float *theta_in, const float *grad_theta_out, const float *grad_logdet,
                           float *grad_theta_in, float *wgrad_partials, float *wgrad, int batch, int L, int mu,
                           int off, int K, int hidden, const float *W1, const float *B1, const float *W2,
                           const float *B2, float slope, void *stream);

/* The inverse coupling layer (no counterpart in the reference), arguments as
 * u1_flow_layer_forward: the same context net (the context plaquettes hold no
 * updated link, so the layer and its inverse see the same parameters), then
 * the inverse mixture transform of each active plaquette by bisection, the
 * link change that undoes a forward step, and logdet[b] = sum of log H' at the
 * solutions (the forward layer's log-det at the returned configuration). */
int u1_flow_layer_inverse(const float *theta_in, float *theta_out, float *logdet, int batch, int L, int mu, int off,
                          int K, int hidden, const float *W1, const float *B1, const float *W2, const float *B2,
                          float slope, void *stream);
/* Backward of u1_flow_layer_inverse (implicit differentiation at the
 * bisection solution), arguments as u1_flow_layer_backward. */
int u1_flow_layer_inverse_backward(const float *theta_in, const float *grad_theta_out, const float *grad_logdet,
                                   float *grad_theta_in, float *wgrad_partials, float *wgrad, int batch, int L,
                                   int mu, int off, int K, int hidden, const float *W1, const float *B1,
                                   const float *W2, const float *B2, float slope, void *stream);

/* Number of kernels this library has launched in the calling process. */
int u1_kernel_launch_count(uint64_t *out);

/* Checked build (libu1b200_check.so, compiled with -DU1_BOUNDS_CHECK; a test
 * build: the reference has none, its kernels run unchecked).  Every link
 * access of the update kernels (single-lattice, batched, measuring and
 * persistent phases) is checked against the (direction, parity) half it
 * addresses and its alignment; a violating access is counted and skipped,
 * never performed.  After every phase a kernel counts the links that were
 * written and also read by another thread, or written twice, in that phase
 * (checkerboard races; not for the persistent variant 4, whose phases
 * overlap within one launch).
 * u1_check_report: out[0] violations, out[1] races, out[2] phases checked,
 * out[3] links accessed (summed over the phases), out[4..6] index, half size
 * and kind (0 read, 1 own read, 2 write) of the first violation (-1: none),
 * out[7] a raced link's buffer offset (-1: none); synchronises the device;
 * reset != 0 clears the counters.  u1_check_selftest runs the checks on a
 * 16-link slab with two refused accesses and two races planted in the marks
 * (never dereferenced) and reports as u1_check_report.  In the normal build
 * both return U1_ERR_UNSUPPORTED. */
int u1_check_report(u1_ctx *ctx, int64_t out[8], int reset);
int u1_check_selftest(u1_ctx *ctx, int64_t out[8]);

#ifdef __cplusplus
}
#endif

#endif /* U1_B200_H */
