"""The explicit-level apply that needs no scratch buffer from its caller (GPU).

Some callers cannot allocate device memory: a host application or language binding that owns
every device allocation and passes this library only pointers, or a loop that must never call
cudaMalloc / cudaFree because they synchronize the device. For them
lpb_apply_explicit_sym_noalloc_f32 keeps its intermediate in an array inside the library. This
test calls it through the C ABI twice in a row on different inputs and compares each result with
lpb_apply_explicit_sym_f32 given a caller-owned scratch buffer (float32 tolerance 2e-5, as the
other float32 operator tests), and checks that a grid beyond its limit is refused.
Runs alone or after the other tests: it builds its own inputs.
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _inputs(dims, seed):
    from loadpath_b200.grid import DevGrid

    g = DevGrid(dims)
    gen = torch.Generator(device="cuda").manual_seed(seed)
    ncp = g.nx * g.ny * g.cpz
    a = torch.randn((ncp, 24, 24), generator=gen, device="cuda")
    k = (a + a.transpose(1, 2)).contiguous()
    cells = g.set_cells(g.cell_field(torch.float32), 1.0)   # zero on the z padding
    k *= cells.reshape(-1, 1, 1)
    mask = g.set_nodes(g.mask_field(), torch.randint(0, 8, (g.NX, g.NY, g.NZ), generator=gen, device="cuda",
                                                     dtype=torch.uint8))
    u = torch.randn(g.node_field(torch.float32).shape, generator=gen, device="cuda")
    bits = torch.stack([((mask >> c) & 1) for c in range(3)]).float()
    u *= bits
    return g, k, u, mask


def test_noalloc_apply_matches_the_scratch_buffer_version_twice():
    from loadpath_b200._lib import lib
    from loadpath_b200.grid import stream_handle

    L = lib()
    st = stream_handle()
    for seed, dims in ((5, (20, 12, 14)), (6, (18, 16, 10))):
        g, k, u, mask = _inputs(dims, seed)
        ncp = g.nx * g.ny * g.cpz
        kp = torch.empty((300, ncp), device="cuda")
        L.lpb_pack_sym_f32(kp.data_ptr(), k.data_ptr(), ncp, st)
        ft = torch.empty((24, ncp), device="cuda")
        want = g.node_field(torch.float32)
        got = g.node_field(torch.float32)
        L.lpb_apply_explicit_sym_f32(want.data_ptr(), u.data_ptr(), kp.data_ptr(), ft.data_ptr(), mask.data_ptr(),
                                     *g.args, st)
        L.lpb_apply_explicit_sym_noalloc_f32(got.data_ptr(), u.data_ptr(), kp.data_ptr(), mask.data_ptr(), *g.args,
                                             st)
        torch.cuda.synchronize()
        w, o = want.cpu().numpy(), got.cpu().numpy()
        assert np.abs(w).max() > 0
        np.testing.assert_allclose(o, w, rtol=2e-5, atol=2e-5 * np.abs(w).max())


def test_noalloc_apply_refuses_grids_beyond_its_limit():
    from loadpath_b200._lib import LpError, lib
    from loadpath_b200.grid import DevGrid, stream_handle

    g = DevGrid((64, 64, 20))          # 64 * 64 * 24 padded cells > 65,536
    dummy = torch.zeros(16, device="cuda")
    with pytest.raises(LpError, match="size beyond"):
        lib().lpb_apply_explicit_sym_noalloc_f32(dummy.data_ptr(), dummy.data_ptr(), dummy.data_ptr(),
                                                 dummy.data_ptr(), *g.args, stream_handle())
