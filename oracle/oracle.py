"""ctypes wrappers of the CPU checkers (TEST INFRASTRUCTURE ONLY).

- Oracle: the FP64 restatement oracle/u1_oracle.cpp (lib/libu1oracle.so).
- Ref:    the reference's own code built in place (oracle/_ref/libu1ref.so,
          see oracle/Makefile and oracle/ref/ref_harness.cu).

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline/reference
legs use this module.  Parity is pinned by tests/test_oracle_pin.py (oracle vs
the reference's own CPU functions, and vs the exact 2D plaquette) and by the
committed fixtures in tests/golden/ (made by tests/golden/make_golden.py from
the reference).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ORACLE_LIB = HERE / "lib" / "libu1oracle.so"
REF_LIB = HERE / "_ref" / "libu1ref.so"
_dp = C.POINTER(C.c_double)


def build(ref: bool = True) -> None:
    """Build the oracle (and, when the reference sources exist at
    $U1_REFERENCE_DIR, oracle/_ref)."""
    targets = ["oracle"] + (["ref"] if ref else [])
    subprocess.run(["make", "-s", "-C", str(HERE), "-j8"] + targets, check=True)


class OGeom(C.Structure):
    _fields_ = [("dims", C.c_int), ("tdir", C.c_int), ("N", C.c_int * 4), ("off", C.c_int * 4),
                ("V", C.c_long), ("Vh", C.c_long), ("Vs", C.c_long), ("beta", C.c_double),
                ("aniso", C.c_double)]


def _arr(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_dp)


class Oracle:
    """FP64 restatement of the reference hot path for one geometry."""

    _lib = None

    @classmethod
    def lib(cls):
        if cls._lib is None:
            if not ORACLE_LIB.exists():
                build(ref=False)
            lib = C.CDLL(str(ORACLE_LIB))
            g = C.POINTER(OGeom)
            sig = {
                "o_setup": (C.c_int, [g, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double]),
                "o_index_eo": (None, [g, C.c_int, C.c_int, C.POINTER(C.c_int)]),
                "o_index_eo_neg": (C.c_long, [g, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int]),
                "o_staple": (None, [g, _dp, C.c_int, C.c_int, C.c_int, _dp]),
                "o_staple_all": (None, [g, _dp, _dp]),
                "o_metropolis_pairs": (C.c_long, [g, _dp, _dp]),
                "o_metropolis_philox": (C.c_long, [g, _dp, C.c_uint64, C.c_uint32, C.c_uint64, C.c_int]),
                "o_philox_uniforms": (None, [g, C.c_uint64, C.c_uint32, C.c_uint64, C.c_int, C.c_int, C.c_int,
                                             C.POINTER(C.c_float)]),
                "o_philox": (None, [C.c_uint32] * 6 + [C.POINTER(C.c_uint32)]),
                "o_overrelax": (None, [g, _dp, C.c_int]),
                "o_metropolis_hits": (C.c_long, [g, _dp, C.c_uint64, C.c_uint32, C.c_uint64, C.c_double, C.c_int,
                                                 C.c_int]),
                "o_phase_hits": (None, [g, _dp, C.c_int, C.c_int, C.c_uint64, C.c_uint32, C.c_uint64, C.c_double,
                                        C.c_int, _dp, _dp]),
                "o_phase": (None, [g, _dp, C.c_int, C.c_int, C.c_int, _dp, C.c_uint64, C.c_uint32, C.c_uint64,
                                   C.c_int, _dp, _dp]),
                "o_hot_start_philox": (None, [g, _dp, C.c_uint64, C.c_uint32, C.c_uint64]),
                "o_plaquette": (None, [g, _dp, _dp]),
                "o_polyakov": (None, [g, _dp, _dp]),
                "o_bessel_ratio": (C.c_double, [C.c_double]),
                "o_fastdiv": (C.c_uint32, [C.c_uint32, C.c_uint32]),
                "o_multihit": (None, [g, _dp, C.c_int, C.c_int, _dp]),
                "o_poly_field": (None, [g, _dp, C.c_int, _dp]),
                "o_poly_corr": (None, [g, _dp, C.c_int, _dp]),
                "o_multilevel": (None, [g, _dp, C.c_uint64, C.c_uint32, C.POINTER(C.c_uint64)] + [C.c_int] * 6
                                 + [_dp]),
                "o_action": (C.c_double, [g, _dp, _dp]),
                "o_topological_charge_2d": (C.c_double, [g, _dp]),
            }
            for name, (ret, args) in sig.items():
                f = getattr(lib, name)
                f.restype = ret
                f.argtypes = args
            cls._lib = lib
        return cls._lib

    def __init__(self, dims: int, N, beta: float, aniso: float = 1.0):
        N = list(N) + [0] * (4 - len(N))
        self.g = OGeom()
        rc = self.lib().o_setup(C.byref(self.g), dims, N[0], N[1], N[2], N[3], beta, aniso)
        if rc != 0:
            raise ValueError("invalid geometry (extents must be even)")
        self.dims = dims
        self.V, self.Vh, self.Vs = self.g.V, self.g.Vh, self.g.Vs
        self.grid = list(self.g.N)
        self.R = self.grid[0] // 2
        self.nlinks = self.V * dims

    def _g(self):
        return C.byref(self.g)

    def index_eo(self, id_: int, parity: int):
        x = (C.c_int * 4)()
        self.lib().o_index_eo(self._g(), id_, parity, x)
        return list(x)

    def index_eo_neg(self, id_, parity, mu, lmu, nu=-1, lnu=0) -> int:
        return int(self.lib().o_index_eo_neg(self._g(), id_, parity, mu, lmu, nu, lnu))

    def staple(self, lat, id_, parity, mu) -> complex:
        o = np.zeros(2)
        self.lib().o_staple(self._g(), _arr(lat), id_, parity, mu, _arr(o))
        return complex(o[0], o[1])

    def staple_all(self, lat) -> np.ndarray:
        """Complex staple of every link, reference layout."""
        o = np.zeros(2 * self.nlinks)
        self.lib().o_staple_all(self._g(), _arr(np.ascontiguousarray(lat)), _arr(o))
        return o[0::2] + 1j * o[1::2]

    def fp32_angle_tolerance(self, lat, base: float = 1e-5) -> np.ndarray:
        """Per-link bound for one FP32 pass vs FP64: base + 2*dS/|S| with
        dS = 12*8 roundings of 2^-24 times the largest staple weight.  The
        reflection theta' = -theta - 2 arg S amplifies a staple error dS by
        2/|S|; links with tiny |S| are ill-conditioned in any precision."""
        w = max(self.g.aniso, 1.0 / self.g.aniso)
        dS = 12 * 8 * 2.0 ** -24 * w
        return base + 2.0 * dS / np.maximum(np.abs(self.staple_all(lat)), 1e-30)

    def metropolis_pairs(self, lat: np.ndarray, pairs: np.ndarray) -> int:
        pairs = np.ascontiguousarray(pairs, dtype=np.float64)
        return int(self.lib().o_metropolis_pairs(self._g(), _arr(lat), _arr(pairs)))

    def metropolis_philox(self, lat, seed, pass_, chain=0, ml=0) -> int:
        return int(self.lib().o_metropolis_philox(self._g(), _arr(lat), seed, chain, pass_, ml))

    def metropolis_hits(self, lat, seed, pass_, delta, nhits, chain=0, ml=0) -> int:
        """One multi-hit windowed Metropolis pass (theta' = theta + delta (2u-1),
        theta' = 2 pi u for delta = 0); returns the number of links moved."""
        return int(self.lib().o_metropolis_hits(self._g(), _arr(lat), seed, chain, pass_, float(delta), int(nhits),
                                                ml))

    def philox_uniforms(self, seed, pass_, parity, mu, chain=0) -> np.ndarray:
        out = np.empty((self.Vh, 2), dtype=np.float32)
        f = (C.c_float * 2)()
        for i in range(self.Vh):
            self.lib().o_philox_uniforms(self._g(), seed, chain, pass_, parity, mu, i, f)
            out[i] = (f[0], f[1])
        return out

    @classmethod
    def philox(cls, ctr, key):
        out = (C.c_uint32 * 4)()
        cls.lib().o_philox(*[int(c) for c in ctr], *[int(k) for k in key], out)
        return [int(v) for v in out]

    def phase(self, lat, met: bool, parity: int, mu: int, pairs=None, seed: int = 0, pass_: int = 0,
              chain: int = 0, ml: int = 0, delta: float = 0.0, nhits: int = 1):
        """One (parity, mu) phase in place; returns (|S| per site, Metropolis
        relative margin 1 - b/exp(dS) per site; with several hits, that of
        the hit closest to its decision).  delta, nhits: the windowed
        multi-hit proposal (defaults: the reference's single whole-circle
        proposal)."""
        smag = np.zeros(self.Vh)
        margin = np.zeros(self.Vh)
        if met and pairs is None and (delta != 0.0 or nhits != 1):
            assert ml == 0
            self.lib().o_phase_hits(self._g(), _arr(lat), parity, mu, seed, chain, pass_, float(delta), int(nhits),
                                    _arr(smag), _arr(margin))
            return smag, margin
        pp = None
        if pairs is not None:
            pairs = np.ascontiguousarray(pairs, dtype=np.float64).reshape(-1)
            assert pairs.size == 2 * self.Vh
            pp = _arr(pairs)
        self.lib().o_phase(self._g(), _arr(lat), int(bool(met)), parity, mu, pp, seed, chain, pass_, ml,
                           _arr(smag), _arr(margin))
        return smag, margin

    def fp32_staple_error(self) -> float:
        """Bound on |S_fp32 - S_fp64|: 2(d-1) plaquette terms of weight up to
        max(xi, 1/xi), each from three float2 links with a few complex
        products, about 12 roundings of 2^-24 per term."""
        w = max(self.g.aniso, 1.0 / self.g.aniso)
        return 2 * (self.dims - 1) * w * 12 * 2.0 ** -24

    def overrelax(self, lat, ml=0) -> None:
        self.lib().o_overrelax(self._g(), _arr(lat), ml)

    def hot_start(self, seed, pass_=0, chain=0) -> np.ndarray:
        lat = np.zeros(self.nlinks)
        self.lib().o_hot_start_philox(self._g(), _arr(lat), seed, chain, pass_)
        return lat

    def update_philox(self, lat, seed, pass_, metrop, ovrn, chain=0, delta=0.0, nhits=1) -> int:
        """metrop Philox Metropolis passes then ovrn OR passes; returns next pass."""
        for m in range(metrop):
            if delta != 0.0 or nhits != 1:
                self.metropolis_hits(lat, seed, pass_ + m, delta, nhits, chain)
            else:
                self.metropolis_philox(lat, seed, pass_ + m, chain)
        for _ in range(ovrn):
            self.overrelax(lat)
        return pass_ + metrop

    def plaquette(self, lat):
        o = np.zeros(4)
        self.lib().o_plaquette(self._g(), _arr(lat), _arr(o))
        return complex(o[0], o[1]), complex(o[2], o[3])

    def polyakov(self, lat) -> complex:
        o = np.zeros(2)
        self.lib().o_polyakov(self._g(), _arr(lat), _arr(o))
        return complex(o[0], o[1])

    @classmethod
    def fastdiv(cls, n: int, d: int) -> int:
        return int(cls.lib().o_fastdiv(n, d))

    @classmethod
    def bessel_ratio(cls, x: float) -> float:
        return float(cls.lib().o_bessel_ratio(x))

    def multihit(self, lat, id_, parity) -> complex:
        o = np.zeros(2)
        self.lib().o_multihit(self._g(), _arr(lat), id_, parity, _arr(o))
        return complex(o[0], o[1])

    def poly_field(self, lat, multihit=False) -> np.ndarray:
        o = np.zeros(2 * self.Vs)
        self.lib().o_poly_field(self._g(), _arr(lat), int(multihit), _arr(o))
        return o[0::2] + 1j * o[1::2]

    def poly_corr(self, lat, multihit=False) -> np.ndarray:
        o = np.zeros(2 * self.R)
        self.lib().o_poly_corr(self._g(), _arr(lat), int(multihit), _arr(o))
        return o[0::2] + 1j * o[1::2]

    def multilevel(self, lat, seed, pass_, n4, k4, n2, k2, metrop, ovrn, chain=0):
        o = np.zeros(2 * self.R)
        p = C.c_uint64(pass_)
        self.lib().o_multilevel(self._g(), _arr(np.ascontiguousarray(lat)), seed, chain, C.byref(p), n4, k4, n2,
                                k2, metrop, ovrn, _arr(o))
        return o[0::2] + 1j * o[1::2], int(p.value)

    def action(self, lat, grad=False):
        if grad:
            gr = np.zeros(self.nlinks)
            s = self.lib().o_action(self._g(), _arr(lat), _arr(gr))
            return float(s), gr
        return float(self.lib().o_action(self._g(), _arr(lat), None))

    def topological_charge_2d(self, lat) -> float:
        return float(self.lib().o_topological_charge_2d(self._g(), _arr(lat)))


class Ref:
    """The reference's own functions (oracle/_ref/libu1ref.so)."""

    _lib = None

    @classmethod
    def available(cls) -> bool:
        return REF_LIB.exists()

    @classmethod
    def lib(cls):
        if cls._lib is None:
            if not REF_LIB.exists():
                raise FileNotFoundError(f"{REF_LIB} not built (needs the reference sources; see oracle/Makefile)")
            lib = C.CDLL(str(REF_LIB))
            i = C.c_int
            sig = {
                "ref_setup_host": (i, [i, i, i, i, i, C.c_double, C.c_double, i, i]),
                "ref_seed_cpu": (None, [i, C.c_uint]),
                "ref_cpu_metropolis": (None, [_dp]),
                "ref_cpu_overrelax": (None, [_dp]),
                "ref_cpu_plaquette": (None, [_dp, _dp]),
                "ref_cpu_polyakov": (None, [_dp, _dp]),
                "ref_record_pairs": (None, [C.c_uint, i, _dp]),
                "ref_index_eo": (None, [i, i, C.POINTER(i)]),
                "ref_index_eo_neg1": (i, [i, i, i, i]),
                "ref_index_eo_neg2": (i, [i, i, i, i, i, i]),
                "ref_host_staple": (None, [_dp, i, i, i, _dp]),
                "ref_host_multihit": (None, [_dp, i, i, _dp]),
                "ref_gpu_start": (i, [i]),
                "ref_gpu_setup": (i, [i, i, i, i, i, C.c_double, C.c_double, i, i]),
                "ref_gpu_update": (C.c_double, [_dp, _dp, i, i, i, i, i]),
                "ref_gpu_measure": (None, [_dp, _dp]),
                "ref_gpu_poly2": (None, [_dp, i, _dp]),
                "ref_gpu_multilevel": (None, [_dp, i, i, i, i, i, i, i, _dp]),
                "ref_gpu_chain": (None, [_dp, i, i, i, i, _dp]),
                "ref_gpu_convert": (None, [_dp, i, _dp]),
                "ref_gpu_plaq_fields": (None, [_dp, i, _dp, _dp]),
            }
            for name, (ret, args) in sig.items():
                f = getattr(lib, name)
                f.restype = ret
                f.argtypes = args
            cls._lib = lib
        return cls._lib

    def __init__(self, dims: int, N, beta: float, aniso: float = 1.0, metrop: int = 1, ovrn: int = 4):
        N = list(N) + [0] * (4 - len(N))
        rc = self.lib().ref_setup_host(dims, N[0], N[1], N[2], N[3], beta, aniso, metrop, ovrn)
        if rc != 0:
            raise ValueError("invalid geometry")
        self.geom = (dims, N, beta, aniso, metrop, ovrn)
        o = Oracle(dims, N, beta, aniso)
        self.V, self.Vh, self.Vs, self.R, self.nlinks = o.V, o.Vh, o.Vs, o.R, o.nlinks
        self.dims = dims

    def seed_cpu(self, nthreads: int, seed: int) -> None:
        self.lib().ref_seed_cpu(nthreads, seed)

    def metropolis(self, lat) -> None:
        self.lib().ref_cpu_metropolis(_arr(lat))

    def overrelax(self, lat) -> None:
        self.lib().ref_cpu_overrelax(_arr(lat))

    def plaquette(self, lat):
        """Reference CPU plaquette: returns (<cos P>, <sin P>) (src/plaquette.cu:32-57)."""
        o = np.zeros(2)
        self.lib().ref_cpu_plaquette(_arr(lat), _arr(o))
        return float(o[0]), float(o[1])

    def polyakov(self, lat) -> complex:
        o = np.zeros(2)
        self.lib().ref_cpu_polyakov(_arr(lat), _arr(o))
        return complex(o[0], o[1])

    def record_pairs(self, seed: int, npass: int) -> np.ndarray:
        out = np.zeros(npass * self.nlinks * 2)
        self.lib().ref_record_pairs(seed, npass, _arr(out))
        return out.reshape(npass, self.nlinks, 2)

    def index_eo(self, id_, parity):
        x = (C.c_int * 4)()
        self.lib().ref_index_eo(id_, parity, x)
        return list(x)

    def index_eo_neg(self, id_, parity, mu, lmu, nu=-1, lnu=0) -> int:
        if nu < 0:
            return int(self.lib().ref_index_eo_neg1(id_, parity, mu, lmu))
        return int(self.lib().ref_index_eo_neg2(id_, parity, mu, lmu, nu, lnu))

    def staple(self, lat, id_, parity, mu) -> complex:
        o = np.zeros(2)
        self.lib().ref_host_staple(_arr(lat), id_, parity, mu, _arr(o))
        return complex(o[0], o[1])

    def multihit(self, lat, id_, parity) -> complex:
        o = np.zeros(2)
        self.lib().ref_host_multihit(_arr(lat), id_, parity, _arr(o))
        return complex(o[0], o[1])


def wrap_diff(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """|a - b| on the circle (radians)."""
    d = np.mod(np.asarray(a) - np.asarray(b) + np.pi, 2 * np.pi) - np.pi
    return np.abs(d)


def env_threads() -> int:
    return int(os.environ.get("U1_CPU_THREADS", os.cpu_count() or 1))
