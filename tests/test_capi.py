"""The C ABI library: builds for sm_100a, loads without a GPU, and exports exactly what
include/loadpath_b200.h declares. CPU only (no kernel is called)."""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

from loadpath_b200 import build
from loadpath_b200._lib import HEADER, LIB_PATH, lib, parse_header


def test_library_builds_and_exports_every_declared_symbol():
    build.build()
    assert os.path.exists(LIB_PATH)
    decls = parse_header()
    names = [d[0] for d in decls]
    assert len(names) == len(set(names))
    out = subprocess.run(["nm", "-D", "--defined-only", LIB_PATH], capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r"\bT (lpb_\w+)", out))
    assert set(names) <= exported, sorted(set(names) - exported)
    # nothing exported that the header does not declare
    assert exported <= set(names), sorted(exported - set(names))
    L = lib()
    assert set(L.fns) == set(names)


def test_header_is_plain_c():
    text = open(HEADER).read()
    assert "torch" not in text and "at::" not in text and "std::" not in text
    # status codes and sizes, the solver handle (an opaque pointer) and its destructor
    for name, ret, types in parse_header():
        if name == "lpb_mg_create":
            assert ret is ctypes.c_void_p
        elif name == "lpb_mg_destroy":
            assert ret is None
        else:
            assert ret in (ctypes.c_int, ctypes.c_longlong), name


def test_modal_ke_pattern_host_only():
    # lpb_modal_ke is host code: the 45 corner-parity coefficients reproduce Ke exactly
    from loadpath_b200.fem import CORNERS, hex8_ke

    s = 2 * CORNERS - 1
    h = np.array([[np.prod([s[k, a] for a in range(3) if (m >> a) & 1]) for k in range(8)] for m in range(8)])
    t = np.kron(h, np.eye(3))
    rows = [3, 3, 3, 4, 4, 5, 5, 6, 6, 7, 7, 7, 8, 8, 9, 9, 10, 10, 11, 11, 11, 12, 12, 13, 13, 14, 14, 14, 15, 15,
            16, 16, 16, 17, 17, 18, 18, 18, 19, 19, 20, 20, 21, 22, 23]
    cols = [3, 7, 14, 4, 6, 5, 12, 4, 6, 3, 7, 14, 8, 13, 9, 20, 10, 17, 11, 16, 18, 5, 12, 8, 13, 3, 7, 14, 15, 19,
            11, 16, 18, 10, 17, 11, 16, 18, 15, 19, 9, 20, 21, 22, 23]
    for el in ("im", "plain"):
        for nu in (0.2, 0.3, 0.45):
            ke = np.ascontiguousarray(hex8_ke(nu, el))
            km = np.zeros(45)
            assert lib().lpb_modal_ke(ke.ctypes.data, km.ctypes.data) == 45
            khat = np.zeros((24, 24))
            khat[rows, cols] = km
            np.testing.assert_allclose(t.T @ khat @ t, ke, rtol=0, atol=1e-14)
    bad = np.random.default_rng(0).standard_normal((24, 24))
    km = np.zeros(45)
    try:
        lib().lpb_modal_ke(np.ascontiguousarray(bad + bad.T).ctypes.data, km.ctypes.data)
        raise AssertionError("a matrix outside the pattern must be rejected")
    except RuntimeError:
        pass


def test_band_layout_host_only():
    """lpb_band_dims (host code): the coarsest level's band numbering puts the longest node axis
    slowest, so the half-bandwidth is 3 (N1 N2 + N2 + 1) + 2 over the two shorter extents."""
    L = lib()
    for cells, (n1, n2) in (((16, 8, 8), (9, 9)), ((8, 16, 8), (9, 9)), ((6, 4, 10), (7, 5)), ((1, 1, 1), (2, 2))):
        out = np.zeros(4, np.int64)
        ntiles = L.lpb_band_dims(*cells, out.ctypes.data)
        n = 3 * int(np.prod(np.asarray(cells) + 1))
        bw = 3 * (n1 * n2 + n2 + 1) + 2
        nt, d = (n + 31) // 32, (bw + 31) // 32
        assert tuple(int(v) for v in out) == (n, nt, d, bw)
        assert ntiles == nt * (d + 1)


def test_mma_scratch_covers_every_reduction():
    """lpb_mma_part_len(m) holds 592 partials for each value of the widest reduction the MMA's
    passes make (prepare M, newton_a 2M + M(M+1)/2, newton_b 4, trial 2 + M): the m = 1 size once
    missed newton_b's four maxima and its partials overran the buffer."""
    from loadpath_b200._lib import lib

    for m in range(1, 9):
        M = 1 if m <= 1 else 2 if m <= 2 else 4 if m <= 4 else 8
        need = 592 * max(M, 2 * M + M * (M + 1) // 2, 4, 2 + M)
        assert lib().lpb_mma_part_len(m) >= need


def test_tuning_table_host_only():
    """lpb_tune_set / lpb_tune_get keep one value per (knob, grid) and clear with 0."""
    from loadpath_b200._lib import LpError, lib

    L = lib()
    assert L.lpb_tune_get(1, 33, 17, 9) == 0
    L.lpb_tune_set(1, 33, 17, 9, 6)
    L.lpb_tune_set(3, 33, 17, 9, 2)
    assert L.lpb_tune_get(1, 33, 17, 9) == 6 and L.lpb_tune_get(3, 33, 17, 9) == 2
    assert L.lpb_tune_get(2, 33, 17, 9) == 0 and L.lpb_tune_get(1, 33, 17, 10) == 0
    L.lpb_tune_set(1, 33, 17, 9, 0)
    assert L.lpb_tune_get(1, 33, 17, 9) == 0
    L.lpb_tune_set(3, 33, 17, 9, 0)
    with pytest.raises(LpError):
        L.lpb_tune_set(9, 33, 17, 9, 1)


def test_tune_candidates():
    from loadpath_b200.tune import candidates

    c = candidates(65, 2)
    assert c[0] == 0 and c[-1] == 65 and all(2 <= z <= 65 for z in c[1:]) and len(c) < 20
    assert candidates(1, 1) == [0, 1]


def test_modal_symmetry_classes_host_only():
    """lpb_modal_sym (host code): the seven classes the fine kernel's product uses rebuild all 45
    corner-parity coefficients of the reference's bricks (plain and incompatible-mode, several
    nu), and the kernel's block formulas give K^ v; coefficients without the symmetry are refused."""
    from loadpath_b200.fem import hex8_ke

    rows = [3, 3, 3, 4, 4, 5, 5, 6, 6, 7, 7, 7, 8, 8, 9, 9, 10, 10, 11, 11, 11, 12, 12, 13, 13, 14, 14, 14, 15, 15,
            16, 16, 16, 17, 17, 18, 18, 18, 19, 19, 20, 20, 21, 22, 23]
    cols = [3, 7, 14, 4, 6, 5, 12, 4, 6, 3, 7, 14, 8, 13, 9, 20, 10, 17, 11, 16, 18, 5, 12, 8, 13, 3, 7, 14, 15, 19,
            11, 16, 18, 10, 17, 11, 16, 18, 15, 19, 9, 20, 21, 22, 23]
    rng = np.random.default_rng(3)
    for el in ("im", "plain"):
        for nu in (0.2, 0.3, 0.45):
            ke = np.ascontiguousarray(hex8_ke(nu, el))
            km = np.zeros(45)
            lib().lpb_modal_ke(ke.ctypes.data, km.ctypes.data)
            cl = np.zeros(7)
            assert lib().lpb_modal_sym(km.ctypes.data, cl.ctypes.data) == 7
            khat = np.zeros((24, 24))
            khat[rows, cols] = km
            amb, b, d, b2, d2, e2, t = cl
            v = rng.standard_normal(24)
            f = np.zeros(24)
            s1 = v[3] + v[7] + v[14]
            for k in (3, 7, 14):
                f[k] = amb * v[k] + b * s1
            for p, q in ((4, 6), (5, 12), (8, 13)):
                f[p] = f[q] = d * (v[p] + v[q])
            s2 = v[11] + v[16] + v[18]
            for k in (11, 16, 18):
                f[k] = b2 * v[k] + b2 * s2
            for p, q in ((9, 20), (10, 17), (15, 19)):
                f[p], f[q] = d2 * v[p] + e2 * v[q], e2 * v[p] + d2 * v[q]
            f[21:] = t * v[21:]
            np.testing.assert_allclose(f, khat @ v, rtol=1e-13, atol=1e-15 * np.abs(khat).max())
    bad = km.copy()
    bad[0] *= 1.01          # one diagonal of the linear normal block off its class
    try:
        lib().lpb_modal_sym(bad.ctypes.data, cl.ctypes.data)
        raise AssertionError("coefficients without the brick's symmetry must be refused")
    except RuntimeError:
        pass


def test_handle_host_helpers_host_only():
    """The host code the solver handle shares with the Python class: numpy's default_rng(seed).random()
    restated (the power iteration's start), the hex8 element, the level-1 Galerkin products and the
    device layout of node and cell fields."""
    import torch

    from loadpath_b200.fem import hex8_ke
    from loadpath_b200.grid import DevGrid
    from oracle import ref_numpy as R

    for seed in (0, 1, 2, 7, 4095):
        got = np.zeros(1000)
        lib().lpb_uniform_numpy(seed, 1000, got.ctypes.data)
        np.testing.assert_array_equal(got, np.random.default_rng(seed).random(1000))
    for inc, el in ((1, "im"), (0, "plain")):
        for nu in (0.2, 0.3, 0.45):
            ke = np.zeros((24, 24))
            lib().lpb_hex8_ke(nu, inc, ke.ctypes.data)
            ref = hex8_ke(nu, el)
            np.testing.assert_allclose(ke, ref, rtol=0, atol=1e-14 * np.abs(ref).max())
            np.testing.assert_array_equal(ke, ke.T)
    ke = np.ascontiguousarray(hex8_ke(0.3, "im"))
    mcat, nkq = np.zeros((8, 576)), np.zeros((64, 576))
    lib().lpb_level1_products(ke.ctypes.data, mcat.ctypes.data, nkq.ctypes.data)
    pk = R.child_prolongations()
    want_m = np.einsum("kai,ab,kbj->kij", pk, ke, pk)
    np.testing.assert_allclose(mcat.reshape(8, 24, 24), want_m, rtol=0, atol=1e-14 * np.abs(want_m).max())
    want_n = np.einsum("kai,qab,kbj->kqij", pk, want_m, pk)
    np.testing.assert_allclose(nkq.reshape(8, 8, 24, 24), want_n, rtol=0, atol=1e-14 * np.abs(want_n).max())
    dims = (6, 4, 10)
    g = DevGrid(dims, device="cpu")
    rng = np.random.default_rng(0)
    nodes = rng.standard_normal(g.node_shape)
    out = np.zeros(g.n_node_field)
    lib().lpb_layout_nodes_f64(np.ascontiguousarray(nodes).ctypes.data, out.ctypes.data, *dims)
    np.testing.assert_array_equal(out, g.nodes_to_dev(nodes, torch.float64).reshape(-1).numpy())
    back = np.zeros(g.node_shape)
    lib().lpb_unlayout_nodes_f64(out.ctypes.data, back.ctypes.data, *dims)
    np.testing.assert_array_equal(back, nodes)
    cells = rng.standard_normal(dims)
    cout = np.zeros(g.cpz // 4 * dims[1] * dims[0] * 4)
    lib().lpb_layout_cells_f64(np.ascontiguousarray(cells).ctypes.data, cout.ctypes.data, *dims)
    np.testing.assert_array_equal(cout, g.cells_to_dev(cells, torch.float64).reshape(-1).numpy())
    sizes = np.zeros(5, np.int64)
    lib().lpb_layout_dims(*dims, sizes.ctypes.data)
    assert list(sizes) == [g.pz, g.cpz, g.n_node_field, g.cpz // 4 * dims[1] * dims[0] * 4, g.pz * g.NY * g.NX]
