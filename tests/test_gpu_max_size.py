"""The largest lattice the row-tiled layout allows: a population array of a 1024 x 1024 x 100 lattice holds
2,032,218,112 elements (19 x padded rows plus guards), just below the 2^31 limit that keeps every index in
32 bits. Size-independent check: the design is invariant along z away from the z walls, so after 4 steps the
planes z = 20 and z = 94 (the highest addresses) must equal plane z = 6 of a 12-deep lattice with the same x-y
cross-section, bit for bit. One plane deeper past the limit is rejected."""
import numpy as np
import pytest
import torch

from xadvcool_b200.lattice import Lattice

pytestmark = pytest.mark.gpu

NX, NY = 1024, 1024


def channel(nz):
    m = np.zeros((NX, NY, nz), np.int32)
    m[:, 0, :] = 1
    m[:, -1, :] = 1
    m[:, :, 0] = 1
    m[:, :, -1] = 1
    for k in range(40):  # square pins through the whole depth
        x0, y0 = 40 + (k * 97) % 900, 30 + (k * 61) % 940
        m[x0:x0 + 12, y0:y0 + 9, 1:-1] = 1
    m[0, 1:-1, 1:-1] = 2
    m[-1, 1:-1, 1:-1] = 3
    return m


def test_largest_lattice_matches_a_thin_slice(cuda):
    kw = dict(tau_fluid=0.6, u_inlet_val=0.05, heat_power=0.1, Pr=7.0, k_ratio=100.0)
    with Lattice(channel(12), **kw) as thin:
        thin.step(4)
        ref = [t[:, :, 6].clone() for t in thin.fields()]
    with Lattice(channel(100), **kw) as big:
        big.step(4)
        fields = big.fields()
        for z in (20, 94):
            for a, b in zip(fields, ref):
                assert torch.equal(a[:, :, z], b), z
        st = big.stats()
    assert st[16] == 0 and np.isfinite(st).all()
    torch.cuda.empty_cache()


def test_past_the_limit_is_rejected(cuda):
    with pytest.raises(Exception, match="too large"):
        Lattice(np.zeros((NX, NY, 106), np.int32), tau_fluid=0.6)
