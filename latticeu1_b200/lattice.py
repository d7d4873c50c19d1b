"""Python host layer over the C ABI: contexts, lattices and counter-based RNGs.

Names mirror the reference's driver surface (reference u1.cpp:44-149):
Context ~ Start/Finalize, Lattice ~ SetupLatticeParameters + Array<double>,
Rng ~ CudaRNG, Lattice.update ~ UpdateLattice, .plaquette ~ Plaquette,
.polyakov ~ Polyakov, .poly_corr ~ Poly2, .multilevel ~ MultiLevel.
All compute runs in the sm_100a kernels of libu1b200.so.
"""
from __future__ import annotations

import ctypes as C
from typing import Sequence

import numpy as np

from ._lib import check, lib, u1_geom


def _grid(dims: int, N: Sequence[int]) -> list[int]:
    """Grid[] as the reference's SetupLatticeParameters builds it
    (reference src/parameters.cu:146-161) from (Nx, Ny, Nz, Nt)."""
    Nx, Ny, Nz, Nt = N
    g = [1, 1, 1, 1]
    g[0] = Nx
    g[1] = Nt if dims == 2 else Ny
    if dims == 3:
        g[2] = Nt
    elif dims > 3:
        g[2] = Nz
    if dims == 4:
        g[3] = Nt
    return g


class Context:
    """One CUDA device (reference Start(gpuid, ...), src/cuda_error_check.cpp:24-45)."""

    def __init__(self, device: int = 0):
        h = C.c_void_p()
        check(lib.u1_ctx_create(int(device), C.byref(h)), "u1_ctx_create")
        self._h = h
        self.device = device

    @property
    def handle(self) -> C.c_void_p:
        return self._h

    def close(self) -> None:
        if self._h:
            lib.u1_ctx_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Rng:
    """Counter-based Philox4x32-10 stream: state = (seed, pass counter)."""

    def __init__(self, ctx: Context, seed: int = 1234):
        h = C.c_void_p()
        check(lib.u1_rng_create(ctx.handle, C.c_uint64(seed), C.byref(h)), "u1_rng_create")
        self._h = h
        self.ctx = ctx

    @property
    def handle(self) -> C.c_void_p:
        return self._h

    @property
    def state(self) -> tuple[int, int]:
        s, p = C.c_uint64(), C.c_uint64()
        check(lib.u1_rng_get_state(self._h, C.byref(s), C.byref(p)), "u1_rng_get_state")
        return int(s.value), int(p.value)

    def set_state(self, seed: int, pass_: int) -> None:
        check(lib.u1_rng_set_state(self._h, C.c_uint64(seed), C.c_uint64(pass_)), "u1_rng_set_state")

    def set_chain(self, chain: int) -> None:
        """Chain number in every Philox counter (independent streams per chain)."""
        check(lib.u1_rng_set_chain(self._h, C.c_uint32(chain)), "u1_rng_set_chain")

    def set_replay(self, pairs: np.ndarray | None) -> None:
        """Shared-stream test mode: pairs[..., 2] = (new theta, b) per link in
        the reference's draw order pass -> parity -> mu -> id."""
        if pairs is None:
            check(lib.u1_rng_set_replay(self._h, None, 0), "u1_rng_set_replay")
            self._replay = None
            return
        arr = np.ascontiguousarray(pairs, dtype=np.float64).reshape(-1, 2)
        self._replay = arr
        check(lib.u1_rng_set_replay(self._h, arr.ctypes.data_as(C.c_void_p), arr.shape[0]), "u1_rng_set_replay")

    def debug_uniforms(self, lat: "Lattice", pass_: int, parity: int, mu: int) -> np.ndarray:
        out = np.empty((lat.Vh, 2), dtype=np.float32)
        check(lib.u1_rng_debug_uniforms(lat.handle, self._h, C.c_uint64(pass_), parity, mu,
                                        out.ctypes.data_as(C.c_void_p)), "u1_rng_debug_uniforms")
        return out

    def close(self) -> None:
        if self._h:
            lib.u1_rng_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Lattice:
    """A U(1) gauge field on the device, float2 links in even/odd SoA order."""

    def __init__(self, ctx: Context, dims: int, N: Sequence[int], beta: float, aniso: float = 1.0):
        N = list(N) + [0] * (4 - len(N))
        geom = u1_geom(dims=int(dims), N=(C.c_int * 4)(*[int(n) for n in N[:4]]),
                       beta=float(beta), aniso=float(aniso))
        h = C.c_void_p()
        check(lib.u1_lattice_create(ctx.handle, C.byref(geom), C.byref(h)), "u1_lattice_create")
        self._h = h
        self.ctx = ctx
        self.dims = int(dims)
        self.beta = float(beta)
        self.aniso = float(aniso)
        info = (C.c_int64 * 8)()
        check(lib.u1_lattice_info(h, info), "u1_lattice_info")
        self.V, self.Vh, self.Vs = int(info[0]), int(info[1]), int(info[2])
        self.grid = [int(info[4 + k]) for k in range(4)]
        self.R = self.grid[0] // 2

    @property
    def handle(self) -> C.c_void_p:
        return self._h

    @property
    def nlinks(self) -> int:
        return self.V * self.dims

    def set_stream(self, stream_ptr: int | None) -> None:
        check(lib.u1_lattice_set_stream(self._h, C.c_void_p(stream_ptr or 0)), "u1_lattice_set_stream")

    def set_coupling(self, beta: float, aniso: float | None = None) -> None:
        aniso = self.aniso if aniso is None else aniso
        check(lib.u1_lattice_set_coupling(self._h, float(beta), float(aniso)), "u1_lattice_set_coupling")
        self.beta, self.aniso = float(beta), float(aniso)

    def set_graphs(self, enable: bool) -> None:
        check(lib.u1_lattice_set_graphs(self._h, int(bool(enable))), "u1_lattice_set_graphs")

    VARIANTS = {0: "auto", 1: "pair32", 2: "pair", 3: "single", 4: "wave", 5: "quad"}

    @property
    def variant(self) -> int:
        v = C.c_int()
        check(lib.u1_lattice_get_variant(self._h, C.byref(v)), "u1_lattice_get_variant")
        return int(v.value)

    def set_variant(self, variant: int) -> None:
        check(lib.u1_lattice_set_variant(self._h, int(variant)), "u1_lattice_set_variant")

    @property
    def block(self) -> int:
        """Threads per block of the phase kernels (tuned with the variant)."""
        v = C.c_int()
        check(lib.u1_lattice_get_block(self._h, C.byref(v)), "u1_lattice_get_block")
        return int(v.value)

    def set_block(self, threads: int) -> None:
        check(lib.u1_lattice_set_block(self._h, int(threads)), "u1_lattice_set_block")

    def set_wave_wait(self, spin_limit: int = 0, stall_tile: int = -1) -> None:
        """Waits of the persistent sweep (variant 4): polls per neighbour wait
        (0: the default) and a tile that never publishes (-1: none)."""
        check(lib.u1_lattice_set_wave_wait(self._h, int(spin_limit), int(stall_tile)), "u1_lattice_set_wave_wait")

    def set_metropolis(self, delta: float = 0.0, nhits: int = 1) -> None:
        """Metropolis proposal: nhits hits per link and pass, each proposing
        theta' = theta + delta (2u - 1), or theta' = 2 pi u for delta = 0
        (the reference's proposal, the default with nhits = 1)."""
        check(lib.u1_lattice_set_metropolis(self._h, float(delta), int(nhits)), "u1_lattice_set_metropolis")

    @property
    def metropolis(self) -> tuple:
        """(delta, nhits) of the Metropolis proposal."""
        d, n = C.c_double(), C.c_int()
        check(lib.u1_lattice_get_metropolis(self._h, C.byref(d), C.byref(n)), "u1_lattice_get_metropolis")
        return float(d.value), int(n.value)

    def tune(self, rng: "Rng") -> int:
        v = C.c_int()
        check(lib.u1_tune(self._h, rng.handle, C.byref(v)), "u1_tune")
        return int(v.value)

    def links_ptr(self) -> int:
        p = C.c_void_p()
        check(lib.u1_lattice_links(self._h, C.byref(p)), "u1_lattice_links")
        return int(p.value)

    def copy_from(self, other: "Lattice") -> None:
        check(lib.u1_lattice_copy(self._h, other.handle), "u1_lattice_copy")

    # -- data movement (reference layout theta[id + p*V/2 + mu*V]) --------
    def import_angles(self, theta) -> None:
        if hasattr(theta, "is_cuda") and theta.is_cuda:
            assert theta.dtype.__str__() == "torch.float64" and theta.numel() == self.nlinks
            check(lib.u1_lattice_import_angles(self._h, C.c_void_p(theta.contiguous().data_ptr()), 1),
                  "u1_lattice_import_angles")
            return
        arr = np.ascontiguousarray(theta, dtype=np.float64).reshape(-1)
        if arr.size != self.nlinks:
            raise ValueError(f"expected {self.nlinks} angles, got {arr.size}")
        check(lib.u1_lattice_import_angles(self._h, arr.ctypes.data_as(C.c_void_p), 0), "u1_lattice_import_angles")

    def export_angles(self, out=None) -> np.ndarray:
        """FP64 angles in the reference layout: into `out` (a CUDA float64
        tensor, or a contiguous float64 host array, e.g. pinned memory) or a
        new numpy array."""
        if out is not None and hasattr(out, "is_cuda") and out.is_cuda:
            check(lib.u1_lattice_export_angles(self._h, C.c_void_p(out.data_ptr()), 1), "u1_lattice_export_angles")
            return out
        if out is not None:
            if hasattr(out, "numpy"):  # host torch tensor (possibly pinned)
                out = out.numpy()
            if out.dtype != np.float64 or not out.flags.c_contiguous or out.size != self.nlinks:
                raise ValueError(f"out must be a contiguous float64 array of {self.nlinks} angles")
            arr = out
        else:
            arr = np.empty(self.nlinks, dtype=np.float64)
        check(lib.u1_lattice_export_angles(self._h, arr.ctypes.data_as(C.c_void_p), 0), "u1_lattice_export_angles")
        return arr

    def _async_buffer(self, buf, what: str):
        """(pointer, on_device) of a caller buffer used by an asynchronous
        copy: no conversion or temporary copy is allowed, since the copy
        reads or writes it after the call returns."""
        if hasattr(buf, "is_cuda"):
            if buf.dtype.__str__() != "torch.float64" or not buf.is_contiguous() or buf.numel() != self.nlinks:
                raise ValueError(f"{what}: need a contiguous float64 tensor of {self.nlinks} angles")
            return C.c_void_p(buf.data_ptr()), int(bool(buf.is_cuda))
        if not isinstance(buf, np.ndarray) or buf.dtype != np.float64 or not buf.flags.c_contiguous \
                or buf.size != self.nlinks:
            raise ValueError(f"{what}: need a contiguous float64 array of {self.nlinks} angles")
        return buf.ctypes.data_as(C.c_void_p), 0

    def import_angles_async(self, theta) -> None:
        """Queue an import on the lattice's stream and return at once.  theta
        (CUDA float64 tensor, or host float64 array / tensor, pinned for an
        asynchronous copy) must stay alive and unchanged until synchronize()."""
        ptr, dev = self._async_buffer(theta, "import_angles_async")
        check(lib.u1_lattice_import_angles_async(self._h, ptr, dev), "u1_lattice_import_angles_async")

    def export_angles_async(self, out) -> None:
        """Queue an export into `out` (as for import_angles_async); the
        angles are there after synchronize()."""
        ptr, dev = self._async_buffer(out, "export_angles_async")
        check(lib.u1_lattice_export_angles_async(self._h, ptr, dev), "u1_lattice_export_angles_async")

    def synchronize(self) -> None:
        check(lib.u1_lattice_synchronize(self._h), "u1_lattice_synchronize")

    # -- Monte Carlo -----------------------------------------------------
    def cold_start(self) -> None:
        check(lib.u1_cold_start(self._h), "u1_cold_start")

    def hot_start(self, rng: Rng) -> None:
        check(lib.u1_hot_start(self._h, rng.handle), "u1_hot_start")

    def update(self, rng: Rng, metrop: int = 1, ovrn: int = 4) -> None:
        check(lib.u1_update(self._h, rng.handle, int(metrop), int(ovrn)), "u1_update")

    def update_measure(self, rng: Rng, metrop: int, ovrn: int, dev_ptr: int) -> None:
        """Sweep whose last pass also measures the plaquettes and the Polyakov
        loop of the final configuration; 6 doubles land at device address
        dev_ptr (asynchronous)."""
        check(lib.u1_update_measure(self._h, rng.handle, int(metrop), int(ovrn), C.c_void_p(dev_ptr)),
              "u1_update_measure")

    def update_phase(self, rng: Rng, metropolis: bool, parity: int, mu: int, hit: int = 0) -> None:
        """One (parity, mu) phase; the rng's pass counter does not advance."""
        check(lib.u1_update_phase(self._h, rng.handle, int(bool(metropolis)), int(parity), int(mu), int(hit)),
              "u1_update_phase")

    # -- measurements ------------------------------------------------------
    def measure(self) -> dict:
        out = (C.c_double * 6)()
        check(lib.u1_measure(self._h, out), "u1_measure")
        return {"plaq_ss": complex(out[0], out[1]), "plaq_st": complex(out[2], out[3]),
                "poly": complex(out[4], out[5])}

    def measure_async(self, dev_ptr: int) -> None:
        check(lib.u1_measure_async(self._h, C.c_void_p(dev_ptr)), "u1_measure_async")

    def plaquette(self) -> tuple[complex, complex]:
        out = (C.c_double * 4)()
        check(lib.u1_plaquette(self._h, out), "u1_plaquette")
        return complex(out[0], out[1]), complex(out[2], out[3])

    def polyakov(self) -> complex:
        out = (C.c_double * 2)()
        check(lib.u1_polyakov(self._h, out), "u1_polyakov")
        return complex(out[0], out[1])

    def poly_corr(self, multihit: bool = False) -> np.ndarray:
        out = (C.c_double * (2 * self.R))()
        check(lib.u1_poly_corr(self._h, int(bool(multihit)), out, 2 * self.R), "u1_poly_corr")
        a = np.frombuffer(out, dtype=np.float64).copy()
        return a[0::2] + 1j * a[1::2]

    def multilevel(self, rng: Rng, n4: int, k4: int, n2: int, k2: int, metrop: int, ovrn: int) -> np.ndarray:
        out = (C.c_double * (2 * self.R))()
        check(lib.u1_multilevel(self._h, rng.handle, n4, k4, n2, k2, metrop, ovrn, out, 2 * self.R),
              "u1_multilevel")
        a = np.frombuffer(out, dtype=np.float64).copy()
        return a[0::2] + 1j * a[1::2]

    # -- formats -----------------------------------------------------------
    def plaquette_fields(self, spacetime: bool = True):
        """(field, means): field is a complex128 CUDA tensor of shape
        (6, V) (spacetime) or (6, V_s) (time averages), components
        (mu,nu) = (0,3),(1,3),(2,3),(1,2),(2,0),(0,1) of 1 - e^{i theta_P},
        natural site order; means holds the six component means."""
        import torch
        n = self.V if spacetime else self.Vs
        field = torch.empty(12 * n, dtype=torch.float64, device=f"cuda:{self.ctx.device}")
        means = (C.c_double * 12)()
        check(lib.u1_plaquette_fields(self._h, int(bool(spacetime)), C.c_void_p(field.data_ptr()), means),
              "u1_plaquette_fields")
        m = np.frombuffer(means, dtype=np.float64).copy()
        return torch.view_as_complex(field.view(6, n, 2)), m[0::2] + 1j * m[1::2]

    def save(self, path, rng: Rng | None = None, exact: bool = True) -> None:
        """Checkpoint: FP64 angles in the reference layout, the rng state and
        (exact) the float2 links for a bit-identical resume."""
        check(lib.u1_checkpoint_save(self._h, rng.handle if rng else None, str(path).encode(), int(bool(exact))),
              "u1_checkpoint_save")

    def load(self, path, rng: Rng | None = None) -> None:
        check(lib.u1_checkpoint_load(self._h, rng.handle if rng else None, str(path).encode()),
              "u1_checkpoint_load")
        g = u1_geom()
        check(lib.u1_checkpoint_info(str(path).encode(), C.byref(g), None, None, None, None),
              "u1_checkpoint_info")
        self.beta, self.aniso = float(g.beta), float(g.aniso)

    def close(self) -> None:
        if self._h:
            lib.u1_lattice_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def checkpoint_info(path) -> dict:
    """Header of a checkpoint through the library (no device work)."""
    g = u1_geom()
    seed, pass_, chain, flags = C.c_uint64(), C.c_uint64(), C.c_uint32(), C.c_uint32()
    check(lib.u1_checkpoint_info(str(path).encode(), C.byref(g), C.byref(seed), C.byref(pass_), C.byref(chain),
                                 C.byref(flags)), "u1_checkpoint_info")
    return {"dims": g.dims, "N": tuple(g.N), "beta": g.beta, "aniso": g.aniso, "seed": seed.value,
            "pass": pass_.value, "chain": chain.value, "flags": flags.value}


def convert_order(theta, dims: int, N: Sequence[int], eo_to_no: bool = True):
    """FP64 angles (CUDA tensor, V*dims) between the even/odd order and the
    natural order theta[lex + mu V], lex = x0 + N0 (x1 + N1 (x2 + N2 x3));
    returns a new tensor (queued on torch's current stream)."""
    import torch
    N = list(N) + [0] * (4 - len(N))
    g = u1_geom(dims=int(dims), N=(C.c_int * 4)(*[int(n) for n in N[:4]]), beta=1.0, aniso=1.0)
    if not (theta.is_cuda and theta.dtype == torch.float64):
        raise ValueError("convert_order: theta must be a float64 CUDA tensor")
    src = theta.contiguous()
    out = torch.empty_like(src)
    with torch.cuda.device(src.device):
        stream = torch.cuda.current_stream(src.device).cuda_stream
        check(lib.u1_convert_order(C.byref(g), C.c_void_p(src.data_ptr()), C.c_void_p(out.data_ptr()),
                                   int(bool(eo_to_no)), C.c_void_p(stream)), "u1_convert_order")
    return out


class Batch:
    """Many independent chains advanced by shared phase launches.

    Chain c follows exactly the trajectory of a single :class:`Lattice`
    driven by an :class:`Rng` with the same seed and ``set_chain(first_chain
    + c)`` through the same hot starts and updates.  ``geoms`` is a list of
    ``(dims, N, beta[, aniso])``; every chain must have the same dims.
    """

    def __init__(self, ctx: Context, geoms: Sequence, seed: int = 1234, first_chain: int = 0):
        n = len(geoms)
        arr = (u1_geom * n)()
        self.shapes = []
        for k, gspec in enumerate(geoms):
            dims, N, beta = int(gspec[0]), list(gspec[1]), float(gspec[2])
            aniso = float(gspec[3]) if len(gspec) > 3 else 1.0
            N = N + [0] * (4 - len(N))
            arr[k] = u1_geom(dims=dims, N=(C.c_int * 4)(*[int(x) for x in N[:4]]), beta=beta, aniso=aniso)
            info = (C.c_int64 * 8)()
            check(lib.u1_geom_validate(C.byref(arr[k]), info), f"u1_geom_validate (chain {k})")
            self.shapes.append((dims, int(info[0])))
        h = C.c_void_p()
        check(lib.u1_batch_create(ctx.handle, n, arr, C.c_uint64(seed), C.c_uint32(first_chain), C.byref(h)),
              "u1_batch_create")
        self._h = h
        self.ctx = ctx
        self.n = n
        self.seed = int(seed)
        self.first_chain = int(first_chain)
        info = (C.c_int64 * 4)()
        check(lib.u1_batch_info(h, info), "u1_batch_info")
        self.dims, self.total_links, self.pair_kernels = int(info[1]), int(info[2]), bool(info[3])

    @property
    def handle(self) -> C.c_void_p:
        return self._h

    def nlinks(self, chain: int) -> int:
        dims, V = self.shapes[chain]
        return dims * V

    @property
    def groups(self) -> int:
        """Chain groups a sweep runs one after another (L2-sized)."""
        v = C.c_int()
        check(lib.u1_batch_groups(self._h, C.byref(v)), "u1_batch_groups")
        return int(v.value)

    def set_stream(self, stream_ptr: int | None) -> None:
        check(lib.u1_batch_set_stream(self._h, C.c_void_p(stream_ptr or 0)), "u1_batch_set_stream")

    @property
    def lanes(self) -> int:
        """Streams a sweep spreads its chain groups over (1 or 2)."""
        v = C.c_int()
        check(lib.u1_batch_get_lanes(self._h, C.byref(v)), "u1_batch_get_lanes")
        return int(v.value)

    def set_lanes(self, lanes: int) -> None:
        check(lib.u1_batch_set_lanes(self._h, int(lanes)), "u1_batch_set_lanes")

    VARIANTS = {5: "quad", 1: "pair32", 3: "single"}

    def tune(self) -> int:
        """Tune (or apply the cached tuning of) the group size and each
        group's kernel and block size; returns the group size in MiB."""
        mb = C.c_int()
        check(lib.u1_batch_tune(self._h, C.byref(mb)), "u1_batch_tune")
        return int(mb.value)

    def configure(self, group_mb: int = 0, choices: Sequence = ()) -> None:
        """Explicit layout: group size in MiB (0: keep) and (variant, threads)
        per group for the first len(choices) groups."""
        n = len(choices)
        v = (C.c_int * max(1, n))(*[int(c[0]) for c in choices])
        t = (C.c_int * max(1, n))(*[int(c[1]) for c in choices])
        check(lib.u1_batch_configure(self._h, int(group_mb), n, v, t), "u1_batch_configure")

    def layout(self) -> list[tuple[int, int, int, int]]:
        """Per group: (first chain, end chain, variant, threads per block)."""
        out = []
        for k in range(self.groups):
            a = (C.c_int * 4)()
            check(lib.u1_batch_group_info(self._h, k, a), "u1_batch_group_info")
            out.append(tuple(int(x) for x in a))
        return out

    def hot_start(self) -> None:
        check(lib.u1_batch_hot_start(self._h), "u1_batch_hot_start")

    def update(self, metrop: int = 1, ovrn: int = 4, measure: bool = False) -> None:
        check(lib.u1_batch_update(self._h, int(metrop), int(ovrn), int(bool(measure))), "u1_batch_update")

    @staticmethod
    def _unpack(a: np.ndarray) -> list[dict]:
        return [{"plaq_ss": complex(r[0], r[1]), "plaq_st": complex(r[2], r[3]), "poly": complex(r[4], r[5])}
                for r in a.reshape(-1, 6)]

    def measure_raw(self) -> np.ndarray:
        out = np.empty(6 * self.n, dtype=np.float64)
        check(lib.u1_batch_measure(self._h, out.ctypes.data_as(C.POINTER(C.c_double))), "u1_batch_measure")
        return out.reshape(self.n, 6)

    def measure(self) -> list[dict]:
        return self._unpack(self.measure_raw())

    def results_raw(self) -> np.ndarray:
        out = np.empty(6 * self.n, dtype=np.float64)
        check(lib.u1_batch_results(self._h, out.ctypes.data_as(C.POINTER(C.c_double))), "u1_batch_results")
        return out.reshape(self.n, 6)

    def results_ptr(self) -> int:
        p = C.c_void_p()
        check(lib.u1_batch_results_device(self._h, C.byref(p)), "u1_batch_results_device")
        return int(p.value)

    def pass_count(self) -> int:
        v = C.c_uint64()
        check(lib.u1_batch_get_pass(self._h, C.byref(v)), "u1_batch_get_pass")
        return int(v.value)

    def import_angles(self, chain: int, theta) -> None:
        arr = np.ascontiguousarray(theta, dtype=np.float64).reshape(-1)
        if arr.size != self.nlinks(chain):
            raise ValueError(f"expected {self.nlinks(chain)} angles, got {arr.size}")
        check(lib.u1_batch_import_angles(self._h, int(chain), arr.ctypes.data_as(C.c_void_p)),
              "u1_batch_import_angles")

    def export_all(self, out=None):
        """All chains' FP64 angles as one CUDA tensor (chain after chain, EO
        layout each); queued on the batch's stream, which the caller orders
        against its own (e.g. by attaching torch's stream with set_stream)."""
        import torch
        if out is None:
            out = torch.empty(self.total_links, dtype=torch.float64, device=f"cuda:{self.ctx.device}")
        check(lib.u1_batch_export_all(self._h, C.c_void_p(out.data_ptr())), "u1_batch_export_all")
        return out

    def export_angles(self, chain: int) -> np.ndarray:
        arr = np.empty(self.nlinks(chain), dtype=np.float64)
        check(lib.u1_batch_export_angles(self._h, int(chain), arr.ctypes.data_as(C.c_void_p)),
              "u1_batch_export_angles")
        return arr

    def close(self) -> None:
        if self._h:
            lib.u1_batch_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
