"""Pin the CPU oracle against golden vectors produced by the upstream numpy code."""

import numpy as np
import pytest

import oracle
from tests.conftest import relerr

TOL = 1e-12


def _cases(index, kind):
    return [c for c in index["cases"] if c["kind"] == kind]


def test_spherical_inverse_forward(golden):
    data, index = golden
    cases = _cases(index, "spherical")
    assert len(cases) > 40
    for c in cases:
        n = c["name"]
        if c["L"] > 64:
            continue
        kw = dict(L=c["L"], spin=c["spin"], nside=c["nside"], sampling=c["sampling"],
                  reality=c["reality"], L_lower=c["L_lower"])
        f = oracle.spherical.inverse(data[f"{n}/flm"], **kw)
        assert relerr(f, data[f"{n}/f"]) < TOL, n
        g = oracle.spherical.forward(data[f"{n}/f"], **kw)
        assert relerr(g, data[f"{n}/flm_fwd"]) < TOL, n


@pytest.mark.slow
def test_spherical_mw_L128(golden):
    data, _ = golden
    kw = dict(L=128, spin=0, sampling="mw")
    f = oracle.spherical.inverse(data["mw_L128/flm"], **kw)
    assert relerr(f, data["mw_L128/f"]) < TOL
    g = oracle.spherical.forward(data["mw_L128/f"], **kw)
    assert relerr(g, data["mw_L128/flm_fwd"]) < TOL
    # round trip of the upstream transform itself
    assert relerr(data["mw_L128/flm_fwd"], data["mw_L128/flm"]) < 1e-10


def test_healpix_iterative_refinement(golden):
    data, index = golden
    for c in _cases(index, "healpix_iter"):
        n = c["name"]
        g = oracle.spherical.forward(data[f"{n}/f"], c["L"], 0, c["nside"], "healpix", True,
                                     iter=c["iter"])
        assert relerr(g, data[f"{n}/flm_fwd"]) < TOL, n


def test_wigner(golden):
    data, index = golden
    for c in _cases(index, "wigner"):
        n = c["name"]
        f = oracle.wigner.inverse(data[f"{n}/flmn"], c["L"], c["N"], None, c["sampling"],
                                  c["reality"])
        assert relerr(f, data[f"{n}/f"]) < TOL, n
        g = oracle.wigner.forward(data[f"{n}/f"], c["L"], c["N"], None, c["sampling"],
                                  c["reality"])
        assert relerr(g, data[f"{n}/flmn_fwd"]) < TOL, n


def test_precompute(golden):
    data, index = golden
    for c in _cases(index, "precompute"):
        n = c["name"]
        L, s, ns, smp = c["L"], c["spin"], c["nside"], c["sampling"]
        kin = oracle.precompute.spin_spherical_kernel(L, s, False, smp, ns, False)
        kfw = oracle.precompute.spin_spherical_kernel(L, s, False, smp, ns, True)
        assert relerr(kin, data[f"{n}/kernel_inv"]) < 1e-11, n
        assert relerr(kfw, data[f"{n}/kernel_fwd"]) < 1e-11, n
        f = oracle.precompute.inverse_transform(data[f"{n}/flm"], kin, L, smp, False, s, ns)
        assert relerr(f, data[f"{n}/f"]) < TOL, n
        g = oracle.precompute.forward_transform(data[f"{n}/f"], kfw, L, smp, False, s, ns)
        assert relerr(g, data[f"{n}/flm_fwd"]) < TOL, n


def test_quadrature(golden):
    data, _ = golden
    for s in ["mwss", "dh", "gl", "healpix"]:
        w = oracle.quadrature.quad_weights_transform(12, s, 0, 4)
        assert relerr(w, data[f"quad/transform_{s}"]) < 1e-14, s
    for s in ["mw", "mwss"]:
        for spin in [0, 1]:
            w = oracle.quadrature.quad_weights(12, s, spin)
            assert relerr(w, data[f"quad/weights_{s}_s{spin}"]) < 1e-14


def test_signal_generator(golden):
    data, _ = golden
    r2 = np.random.default_rng(8966433580120847635)
    np.testing.assert_array_equal(oracle.signal.generate_flm(r2, 9, 0, 1, False),
                                  data["gen/flm_L9_s1"])
    np.testing.assert_array_equal(oracle.signal.generate_flm(r2, 9, 2, 0, True),
                                  data["gen/flm_L9_real"])
    np.testing.assert_array_equal(oracle.signal.generate_flmn(r2, 6, 3, 0, False),
                                  data["gen/flmn_L6_N3"])
    np.testing.assert_array_equal(oracle.signal.generate_flmn(r2, 6, 3, 0, True),
                                  data["gen/flmn_L6_N3_real"])


def test_rotation_matches_upstream_risbo():
    """oracle.rotation against upstream's own Risbo recursion and rotate_flms contraction
    (tests/golden/make_rotation.py)."""
    import os

    from tests.conftest import GOLDEN_DIR

    d = np.load(os.path.join(GOLDEN_DIR, "rotation.npz"))
    for k in range(3):
        L = int(d[f"r{k}/L"])
        rot = tuple(d[f"r{k}/rotation"])
        dl = oracle.rotation.generate_rotate_dls(L, rot[1])
        assert np.abs(dl - d[f"r{k}/dls"]).max() < 1e-13
        r = oracle.rotation.rotate_flms(d[f"r{k}/flm"], L, rot)
        assert np.abs(r - d[f"r{k}/rotated"]).max() < 1e-13 * np.abs(d[f"r{k}/rotated"]).max()


def _fw_golden():
    import json
    import os

    from tests.conftest import GOLDEN_DIR

    d = np.load(os.path.join(GOLDEN_DIR, "fourier_wigner.npz"))
    with open(os.path.join(GOLDEN_DIR, "fourier_wigner.json")) as fh:
        return d, json.load(fh)["cases"]


def test_fourier_wigner_matches_upstream():
    """oracle.fourier_wigner against upstream's numpy Fourier-Wigner transforms and
    fourier_wigner_kernel (tests/golden/make_fourier_wigner.py), atol 1e-12 as upstream's
    tests/test_fourier_wigner.py."""
    fw = oracle.fourier_wigner
    d, cases = _fw_golden()
    for L in (8, 16):
        delta, quads = fw.fourier_wigner_kernel(L)
        assert np.abs(delta - d[f"kernel_L{L}/delta"]).max() < 1e-13
        assert np.abs(quads - d[f"kernel_L{L}/quads"]).max() < 1e-13
    seen = 0
    for c in cases:
        if c["kind"] != "fourier_wigner":
            continue
        n, L, N, s, r = c["name"], c["L"], c["N"], c["sampling"], c["reality"]
        f = fw.inverse_transform(d[f"{n}/flmn"], L, N, None, r, s)
        np.testing.assert_allclose(f, d[f"{n}/f"], atol=1e-12)
        g = fw.forward_transform(d[f"{n}/f"], L, N, None, r, s)
        np.testing.assert_allclose(g, d[f"{n}/flmn_fwd"], atol=1e-12)
        # the forward inverts the inverse on band-limited inputs
        np.testing.assert_allclose(d[f"{n}/flmn_fwd"], d[f"{n}/flmn"], atol=1e-12)
        seen += 1
    assert seen == 10


def test_spin_subset_ops_match_upstream():
    """wigner_subset_to_s2 / s2_to_wigner_subset / so3_to_wigner_subset against upstream
    custom_ops (batch 2, channels 3, mixed spins)."""
    fw = oracle.fourier_wigner
    d, cases = _fw_golden()
    for c in cases:
        if c["kind"] != "subset_ops":
            continue
        n, L, N, s, sp = c["name"], c["L"], c["N"], c["sampling"], np.array(c["spins"])
        DW = fw.fourier_wigner_kernel(L)
        np.testing.assert_allclose(fw.wigner_subset_to_s2(d[f"{n}/flmn"], sp, DW, L, s),
                                   d[f"{n}/fs"], atol=1e-12)
        np.testing.assert_allclose(fw.s2_to_wigner_subset(d[f"{n}/fs"], sp, DW, L, s),
                                   d[f"{n}/back"], atol=1e-12)
        np.testing.assert_allclose(fw.so3_to_wigner_subset(d[f"{n}/fso3"], sp, DW, L, N, s),
                                   d[f"{n}/sub"], atol=1e-12)
    with pytest.raises(ValueError):
        fw.wigner_subset_to_s2(d["ops0/flmn"], np.array([0, 1]), DW, 8, "mw")
    with pytest.raises(ValueError):
        fw.inverse_transform(d["fw0/flmn"], 8, 2, None, False, "gl")
