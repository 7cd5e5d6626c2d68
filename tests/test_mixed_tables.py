"""CPU checks of the mixed form's own operator tables (fmmg_operator 5 and 6)
against independent numpy computations on host-only handles.

Table 5 is the M2L translation spectrum on the (2np-1)^3 grid: the kernel from
a source at 2*(i1, i2, i3) sampled at the grid offsets (i < np ? i : i - n)
steps of 2/(np-1) per axis and r2c transformed -- the construction of
fmm3d_mpi/matmgnt3d_mpi.cpp:385-411 on the odd grid.  A replaced (2np)^3
spectrum (table 4) is converted exactly: inverse transform, keep the offsets
-(np-1)..np-1, forward transform on the odd grid.  Table 6 is the parent
upward operator pinv(UC->UE) x M2M with the 8 octants side by side.  The
operator sets a process keeps are shared between handles.
"""
import numpy as np
import pytest

import fmmg
import oracle as O

MM = {111: 111, 121: 111, 301: 301, 311: 301, 312: 111, 321: 301, 322: 111, 511: 511, 521: 511}
COEFS = (1.0, 0.25)


def _handle(kt, np_):
    rng = np.random.default_rng(3)
    src = rng.random((300, 3))
    f = fmmg.FMM3d(kt, np_=np_, pts_max=60, device=-1)
    f.setup(src, src, src)
    return f


def _translations():
    return [(a, b, c) for a in range(-3, 4) for b in range(-3, 4) for c in range(-3, 4)
            if max(abs(a), abs(b), abs(c)) > 1]


def _dofs(kt):
    m = MM[kt]
    return O.src_dof(m), O.trg_dof(m)


def _sampled_spectrum(kt, np_, n, t):
    """rfftn of the equivalent kernel sampled on the n^3 grid, [kz][ky][kx][h]."""
    sdm, tdm = _dofs(kt)
    off = np.array([(i if i < np_ else i - n) * 2.0 / (np_ - 1) for i in range(n)])
    z, y, x = np.meshgrid(off, off, off, indexing="ij")
    reg = np.stack([x.ravel(), y.ravel(), z.ravel()], 1)
    sp = 2.0 * np.array([t], dtype=np.float64)
    K = O.kernel_matrix(MM[kt], sp, sp, reg, COEFS)  # (n^3 tdm) x sdm
    grid = K.reshape(n ** 3, tdm, sdm).transpose(0, 2, 1).reshape(n, n, n, sdm * tdm)
    return np.fft.rfftn(grid, axes=(0, 1, 2))


def _as_complex(v, n, mdof):
    return v.view(np.complex128).reshape(n, n, n // 2 + 1, mdof)


def _to_odd_grid(X, np_):
    """Exact conversion of a (2np)^3 half spectrum to the (2np-1)^3 grid."""
    n, m = 2 * np_, 2 * np_ - 1
    g = np.fft.irfftn(X, s=(n, n, n), axes=(0, 1, 2))
    keep = [i if i < np_ else i - m + n for i in range(m)]
    return np.fft.rfftn(g[np.ix_(keep, keep, keep)], axes=(0, 1, 2))


@pytest.mark.parametrize("kt,np_", [(111, 4), (111, 6), (321, 4), (511, 3)])
def test_odd_grid_spectra_are_sampled_kernel_transforms(kt, np_):
    f = _handle(kt, np_)
    sdm, tdm = _dofs(kt)
    tr = _translations()
    for idx in (0, 57, 200, 315):
        # the helper reproduces table 4 on the even grid ...
        ref4 = _sampled_spectrum(kt, np_, 2 * np_, tr[idx])
        got4 = _as_complex(f.operator(4, idx), 2 * np_, sdm * tdm)
        np.testing.assert_allclose(got4, ref4, rtol=0, atol=1e-12 * np.abs(ref4).max())
        # ... and table 5 on the odd one
        ref5 = _sampled_spectrum(kt, np_, 2 * np_ - 1, tr[idx])
        got5 = _as_complex(f.operator(5, idx), 2 * np_ - 1, sdm * tdm)
        np.testing.assert_allclose(got5, ref5, rtol=0, atol=1e-12 * np.abs(ref5).max())
        # the odd grid is the even one restricted to the offsets it keeps
        np.testing.assert_allclose(_to_odd_grid(ref4, np_), ref5, rtol=0, atol=1e-12 * np.abs(ref5).max())


@pytest.mark.parametrize("kt,np_", [(111, 5), (311, 4)])
def test_replaced_spectrum_is_converted_exactly(kt, np_):
    f = _handle(kt, np_)
    sdm, tdm = _dofs(kt)
    n, mdof = 2 * np_, sdm * tdm
    # a translation given another's spectrum takes that one's odd-grid spectrum
    a11, b = f.operator(4, 11), f.operator(4, 300)
    b5 = f.operator(5, 300)
    f.set_operator(4, 10, b)
    np.testing.assert_allclose(f.operator(5, 10), b5, rtol=0, atol=1e-12 * np.abs(b5).max())
    # an arbitrary real-grid spectrum follows the numpy conversion
    rng = np.random.default_rng(7)
    X = np.fft.rfftn(rng.standard_normal((n, n, n, mdof)), axes=(0, 1, 2))
    f.set_operator(4, 57, X.view(np.float64).ravel())
    np.testing.assert_allclose(_as_complex(f.operator(4, 57), n, mdof), X, rtol=0, atol=0)
    want = _to_odd_grid(X, np_)
    got = _as_complex(f.operator(5, 57), n - 1, mdof)
    np.testing.assert_allclose(got, want, rtol=0, atol=1e-12 * np.abs(want).max())
    # the untouched translations keep their tables
    np.testing.assert_array_equal(f.operator(4, 300), b)
    np.testing.assert_array_equal(f.operator(4, 11), a11)


@pytest.mark.parametrize("kt,np_", [(111, 4), (111, 6), (311, 4), (521, 4)])
def test_folded_upward_operator_is_pinv_times_m2m(kt, np_):
    f = _handle(kt, np_)
    # table 0 is (ue x uc), table 1 octants (uc x ue), table 6 (ue x 8 ue),
    # all column-major
    pinv, fold = f.operator(0), f.operator(6)
    ue = int(round(np.sqrt(fold.size / 8)))
    uc = pinv.size // ue
    assert fold.size == 8 * ue * ue and pinv.size == ue * uc
    R = pinv.reshape(uc, ue).T
    want = np.hstack([R @ f.operator(1, o).reshape(ue, uc).T for o in range(8)])
    got = fold.reshape(8 * ue, ue).T
    eps = 0.1 ** (np_ + 1)
    np.testing.assert_allclose(got, want, rtol=0, atol=100 * 1e-16 / eps * np.abs(want).max())
    # a replaced pseudo-inverse is refactored into the fold
    f.set_operator(0, 0, 0.5 * pinv)
    np.testing.assert_allclose(f.operator(6).reshape(8 * ue, ue).T, 0.5 * want, rtol=0,
                               atol=100 * 1e-16 / eps * np.abs(want).max())
    # and a replaced octant enters its block only
    M3 = f.operator(1, 3)
    f.set_operator(1, 3, 2.0 * M3)
    g2 = f.operator(6).reshape(8 * ue, ue).T
    want2 = 0.5 * want.copy()
    want2[:, 3 * ue:4 * ue] *= 2.0
    np.testing.assert_allclose(g2, want2, rtol=0, atol=100 * 1e-16 / eps * np.abs(want).max())


def test_mixed_tables_are_read_only():
    f = _handle(111, 4)
    with pytest.raises(fmmg.FmmgError):
        f.set_operator(5, 0, f.operator(5, 0))
    with pytest.raises(fmmg.FmmgError):
        f.set_operator(6, 0, f.operator(6))
    with pytest.raises(fmmg.FmmgError):
        f.operator(5, 316)


def test_operator_sets_are_shared_between_handles_not_their_replacements():
    """A process keeps the operator sets it built (the reference shares one
    operator manager per kernel and order, fmm3d_mpi/matmgnt3d_mpi.cpp:526-543):
    a second handle gets bit-identical tables; a table one handle replaces stays
    its own, and a new setup of that handle resets it."""
    a = _handle(111, 5)
    b = _handle(111, 5)
    for which, idx in ((0, 0), (1, 3), (2, 0), (3, 5), (4, 100), (5, 100), (6, 0)):
        np.testing.assert_array_equal(a.operator(which, idx), b.operator(which, idx))
    orig = a.operator(0)
    a.set_operator(0, 0, 2.0 * orig)
    np.testing.assert_array_equal(_handle(111, 5).operator(0), orig)
    np.testing.assert_array_equal(a.operator(0), 2.0 * orig)
    rng = np.random.default_rng(5)
    a.setup(rng.random((400, 3)))
    np.testing.assert_array_equal(a.operator(0), orig)
    # a handle with no replaced table keeps its own tables through new setups
    before = [b.operator(w, i) for w, i in ((0, 0), (1, 7), (3, 2), (4, 315), (5, 0), (6, 0))]
    b.setup(rng.random((500, 3)))
    b.setup(rng.random((600, 3)))
    after = [b.operator(w, i) for w, i in ((0, 0), (1, 7), (3, 2), (4, 315), (5, 0), (6, 0))]
    for x, y in zip(before, after):
        np.testing.assert_array_equal(x, y)
    # other coefficients are another set (Navier's Poisson ratio enters the kernel)
    n1 = fmmg.FMM3d(511, np_=3, pts_max=60, coefs=(1.0, 0.25), device=-1)
    n2 = fmmg.FMM3d(511, np_=3, pts_max=60, coefs=(1.0, 0.3), device=-1)
    assert not np.array_equal(n1.operator(1, 0), n2.operator(1, 0))


def test_operator_sets_under_concurrent_creation():
    """Handles created from several threads at once (the foreign calls run
    without the interpreter lock) get the same tables as handles created one
    at a time, also while the process's sets are evicted (more keys than it
    keeps)."""
    import threading
    keys = [(111, 3), (111, 4), (121, 5), (312, 3), (111, 3), (511, 3), (111, 4), (321, 3)]
    ref = {}
    for kt, np_ in set(keys):
        f = fmmg.FMM3d(kt, np_=np_, pts_max=60, device=-1)
        ref[(kt, np_)] = [f.operator(w, i) for w, i in ((0, 0), (2, 0), (4, 7), (5, 300), (6, 0))]
    got, errors = {}, []

    def make(j, kt, np_):
        try:
            f = fmmg.FMM3d(kt, np_=np_, pts_max=60, device=-1)
            got[j] = ((kt, np_), [f.operator(w, i) for w, i in ((0, 0), (2, 0), (4, 7), (5, 300), (6, 0))])
        except Exception as e:  # reported below
            errors.append(e)

    for _ in range(2):
        th = [threading.Thread(target=make, args=(j, kt, np_)) for j, (kt, np_) in enumerate(keys)]
        for t in th:
            t.start()
        for t in th:
            t.join()
        assert not errors, errors
        for j, (key, tabs) in got.items():
            for a, b in zip(tabs, ref[key]):
                np.testing.assert_array_equal(a, b)


def test_failed_setup_leaves_a_handle_usable():
    """A setup refused for its input (a point outside the root box) changes
    nothing; the next valid setup of the same handle builds the same plan and
    keeps the same tables as a fresh handle."""
    rng = np.random.default_rng(9)
    x = rng.random((800, 3))
    f = _handle(321, 4)
    tabs = [f.operator(w, i) for w, i in ((0, 0), (2, 0), (4, 9), (6, 0))]
    bad = x.copy()
    bad[17, 1] = 1.5
    with pytest.raises(fmmg.FmmgError):
        f.setup(bad, bad)
    f.setup(x, x)
    g = fmmg.FMM3d(321, np_=4, pts_max=60, device=-1)
    g.setup(x, x)
    for a, b in zip(f.tree(), g.tree()):
        np.testing.assert_array_equal(a, b)
    for which in range(4):
        for a, b in zip(f.lists(which), g.lists(which)):
            np.testing.assert_array_equal(a, b)
    for t, (w, i) in zip(tabs, ((0, 0), (2, 0), (4, 9), (6, 0))):
        np.testing.assert_array_equal(f.operator(w, i), t)
