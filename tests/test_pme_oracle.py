"""The oracle's smooth-PME restatement (Essmann et al. 1995) against the
oracle's Ewald sum, which is pinned to the reference (forcefield/ewald.cpp):
the reciprocal energy, virial and forces converge to the k-vector sum as the
grid and the B-spline order grow.  No GPU."""
import numpy as np
import pytest

import oracle as O
from conftest import load_golden

SPCE = load_golden("nist_spce.npz")


def ewald_recip(c, alpha, kmax=12):
    pos, box = SPCE[f"pos{c}"], SPCE[f"box{c}"]
    q = np.where(SPCE[f"isO{c}"], -0.8476, 0.4238)
    mol = np.arange(len(q)) // 3
    f1, t1, w1 = O.ewald(pos, box, q, mol, kmax=kmax, alpha=alpha)
    f0, t0, w0 = O.ewald(pos, box, q, mol, kmax=0, alpha=alpha)
    return t1["reciprocal"], w1 - w0, f1 - f0, pos, box, q


@pytest.mark.parametrize("c", [1, 4])
def test_pme_converges_to_the_ewald_sum(c):
    alpha = 5.6 / SPCE[f"box{c}"].min()
    e_ref, w_ref, f_ref, pos, box, q = ewald_recip(c, alpha)
    errors = []
    for K, p in ((16, 4), (24, 6), (32, 6), (48, 8)):
        K = int(np.ceil(K * box[0] / 20.0))  # the same spacing for larger boxes
        e, w, f = O.pme_recip(pos, box, q, alpha, K, p)
        errors.append((abs(e - e_ref) / abs(e_ref), abs(w - w_ref) / abs(w_ref),
                       np.sqrt(np.mean((f - f_ref) ** 2) / np.mean(f_ref ** 2))))
    errors = np.array(errors)
    assert np.all(np.diff(errors, axis=0) < 0)  # every refinement helps every quantity
    assert errors[-1, 0] < 1e-8 and errors[-1, 1] < 1e-7 and errors[-1, 2] < 1e-7


def test_bspline_partition_of_unity_and_derivatives():
    w = np.linspace(0.0, 0.999, 37)
    for p in (4, 6, 8):
        c, d = O._bspline_weights(w, p)
        assert np.allclose(c.sum(axis=1), 1.0, atol=1e-14)
        assert np.allclose(d.sum(axis=1), 0.0, atol=1e-13)
        h = 1e-6
        cp, _ = O._bspline_weights(np.clip(w + h, 0, 1 - 1e-12), p)
        cm, _ = O._bspline_weights(np.clip(w - h, 0, 1), p)
        inner = (w > 2 * h) & (w < 1 - 2 * h)
        assert np.allclose(((cp - cm) / (2 * h))[inner], d[inner], atol=1e-7)


def test_pme_converges_in_a_non_cubic_box():
    """Configuration 1 stretched by (1, 1.25, 1.1): unequal grids per axis at
    about the same spacing converge to the Ewald sum as in a cubic box."""
    scale = np.array([1.0, 1.25, 1.1])
    pos, box = SPCE["pos1"] * scale, SPCE["box1"] * scale
    q = np.where(SPCE["isO1"], -0.8476, 0.4238)
    mol = np.arange(len(q)) // 3
    alpha = 0.3
    f1, t1, w1 = O.ewald(pos, box, q, mol, kmax=14, alpha=alpha)
    f0, t0, w0 = O.ewald(pos, box, q, mol, kmax=0, alpha=alpha)
    e_ref, f_ref = t1["reciprocal"], f1 - f0
    errs = []
    for h, p in ((1.25, 4), (0.8, 6), (0.5, 8)):
        K = [int(np.ceil(L / h)) for L in box]
        e, w, f = O.pme_recip(pos, box, q, alpha, K, p)
        errs.append((abs(e - e_ref) / abs(e_ref), np.sqrt(np.mean((f - f_ref) ** 2) / np.mean(f_ref ** 2))))
    errs = np.array(errs)
    assert np.all(np.diff(errs, axis=0) < 0)
    assert errs[-1, 0] < 1e-8 and errs[-1, 1] < 1e-7


def test_fft_friendly_grid_sizes():
    import moleculardynamics_b200 as md
    assert [md.fft_size(k) for k in (1, 7, 11, 13, 47, 49.72, 63, 97, 121)] == \
        [1, 7, 12, 14, 48, 50, 63, 98, 125]
