"""Maximum lattice size: the link index id + parity*V/2 + mu*V is a 32-bit
int, so u1_lattice_create accepts V*dims <= 2^31 links and refuses more.
At exactly 2^31 links (4D 128^3 x 256, 17.2 GB of float2 links) the GPU
path is checked through properties that do not need the FP64 oracle:

  * an overrelaxation phase is an involution (the staple of a link does not
    depend on the links of its own (parity, mu) block), so applying it twice
    restores every link to FP32 rounding;
  * overrelaxation conserves the total action, so after a whole OR pass
    n_SS <1 - P_SS> + n_ST <1 - P_ST> (isotropic, 3 + 3 planes in 4D) is
    unchanged to FP32 rounding, while the spatial/temporal split moves (the
    FP64 oracle shows the same exchange on small lattices);
  * the measurement taken from the sweep's last pass equals a separate
    measurement of the final configuration.
"""
import ctypes as C

import pytest

from latticeu1_b200._lib import lib, u1_geom

MAX_GEOM = (128, 128, 128, 256)  # V * 4 = 2^31
U1_ERR_UNSUPPORTED = -3


def _validate(dims, N):
    g = u1_geom(dims, (C.c_int * 4)(*N), 1.0, 1.0)
    out = (C.c_int64 * 8)()
    return lib.u1_geom_validate(C.byref(g), out), list(out)


def test_geom_limit_is_2_pow_31_links():
    rc, out = _validate(4, MAX_GEOM)
    assert rc == 0 and out[0] * 4 == 2 ** 31
    assert _validate(4, (128, 128, 128, 258))[0] == U1_ERR_UNSUPPORTED
    assert _validate(3, (1024, 1024, 0, 1024))[0] == U1_ERR_UNSUPPORTED  # 2^30 sites x 3 links
    assert _validate(2, (32768, 0, 0, 32768))[0] == 0  # 2^30 sites x 2 links = 2^31


class _DeviceArray:
    """float32 view of device memory for torch.as_tensor."""

    def __init__(self, ptr, n):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": "<f4", "data": (ptr, False), "version": 3}


def _action(m):
    return m["plaq_ss"].real + m["plaq_st"].real  # 3 SS + 3 ST planes, equal weights at xi = 1


@pytest.mark.gpu
def test_max_size_or_involution_action_and_fused_measurement(ctx):
    import torch
    from latticeu1_b200 import Lattice, Rng
    lat = Lattice(ctx, 4, MAX_GEOM, 1.0)
    assert lat.nlinks == 2 ** 31
    rng = Rng(ctx, 11)
    lat.hot_start(rng)
    links = torch.as_tensor(_DeviceArray(lat.links_ptr(), 2 * lat.nlinks), device="cuda")
    # one OR phase twice: identity to rounding, on every link of the block
    before = links.clone()
    for p, mu in [(0, 0), (1, 3)]:
        lat.update_phase(rng, False, p, mu)
        lat.update_phase(rng, False, p, mu)
        torch.cuda.synchronize()
        worst = 0.0
        for a, b in zip(links.split(1 << 28), before.split(1 << 28)):
            worst = max(worst, float((a - b).abs().max()))
        assert worst < 2e-6, (p, mu, worst)
    del before
    torch.cuda.empty_cache()
    # whole OR passes conserve the total action (from a hot and from a moved configuration)
    for _ in range(2):
        m0 = lat.measure()
        lat.update(rng, 0, 1)
        m1 = lat.measure()
        assert abs(_action(m1) - _action(m0)) < 1e-6, (m0, m1)
        lat.update(rng, 1, 1)
    # the measured sweep equals a separate measurement
    out = torch.zeros(6, dtype=torch.float64, device="cuda")
    lat.update_measure(rng, 1, 1, out.data_ptr())
    torch.cuda.synchronize()
    got, want = out.cpu().numpy(), lat.measure()
    assert abs(complex(got[0], got[1]) - want["plaq_ss"]) < 2e-6
    assert abs(complex(got[2], got[3]) - want["plaq_st"]) < 2e-6
    assert abs(complex(got[4], got[5]) - want["poly"]) < 2e-6
    assert abs(_action(want) - _action(m1)) > 1e-3  # the Metropolis passes moved it
    lat.close()
