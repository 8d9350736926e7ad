"""Build the committed golden fixtures from the reference's own test data.

Reads the reference's Julia-generated ground-truth arrays
(zaneblood1/CMBLensing.py ``tests/ground_truth_data``, 256x256, 2.5 arcmin
pixels, seed 67, 7 RK4 steps) and writes compact ``.npz`` fixtures next to
this script:

* inputs (fields, phi, operator diagonals) are stored in full, float64 /
  complex128, compressed;
* outputs (lensed / adjoint-lensed fields, gradients) are stored as a seeded
  subsample of 8192 entries plus the row/column indices, so the fixtures stay
  small while still pinning every output;
* logpdf scalars are stored exactly;
* ``mix.npz`` holds the mixing diagonals D (T, EE, BB) and G, the
  quadratic-estimate noise Nphi (T and QU sets) and the subsampled mixed phi
  gradients (T-only and QU-only sets).

Run once in a container that has the reference checked out::

    python tests/golden/make_golden.py /path/to/CMBLensing.py/tests/ground_truth_data

The tests never read the reference tree; they only read these fixtures.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
NSUB = 8192


def _sub_index(shape, seed):
    rng = np.random.default_rng(seed)
    flat = rng.choice(shape[0] * shape[1], size=NSUB, replace=False)
    flat.sort()
    return np.stack(np.unravel_index(flat, shape), axis=0).astype(np.int32)


def main(src):
    L = lambda name: np.load(os.path.join(src, name))
    meta = dict(nside=int(open(os.path.join(src, "n_side.txt")).read().strip()),
                theta_pix=float(open(os.path.join(src, "theta_pix.txt")).read().strip()))
    shape = L("phi_I.npz").shape
    idx = _sub_index(shape, 67)

    def sub(name):
        return L(name)[idx[0], idx[1]]

    # lensing: inputs in full, outputs subsampled
    np.savez_compressed(os.path.join(HERE, "lens_I.npz"), idx=idx, **meta,
                        phi=L("phi_I.npz"), t=L("t_field_I.npz"),
                        t_lensed=sub("t_lensed_field_I.npz"), t_adjoint=sub("t_adjoint_lensed_field_I.npz"))
    np.savez_compressed(os.path.join(HERE, "lens_P.npz"), idx=idx, **meta,
                        phi=L("phi_P.npz"), e=L("e_field_P.npz"), b=L("b_field_P.npz"),
                        e_lensed=sub("e_lensed_field_P.npz"), b_lensed=sub("b_lensed_field_P.npz"),
                        e_adjoint=sub("e_adjoint_lensed_field_P.npz"), b_adjoint=sub("b_adjoint_lensed_field_P.npz"))
    np.savez_compressed(os.path.join(HERE, "lens_IP.npz"), idx=idx, **meta,
                        phi=L("phi_IP.npz"), t=L("t_field_IP.npz"), e=L("e_field_IP.npz"), b=L("b_field_IP.npz"),
                        t_lensed=sub("t_lensed_field_IP.npz"), e_lensed=sub("e_lensed_field_IP.npz"),
                        b_lensed=sub("b_lensed_field_IP.npz"), t_adjoint=sub("t_adjoint_lensed_field_IP.npz"),
                        e_adjoint=sub("e_adjoint_lensed_field_IP.npz"), b_adjoint=sub("b_adjoint_lensed_field_IP.npz"))
    # inference goldens: logpdf, gradf, grad_phi (T-only and QU-only sets)
    np.savez_compressed(os.path.join(HERE, "infer_I.npz"), idx=idx, **meta,
                        data_t=L("data_t_field_I.npz"), cn=L("cn_I.npz"), cf=L("cf_I.npz"), cphi=L("cphi_I.npz"),
                        m=L("m_I.npz"), b=L("b_I.npz"),
                        gradf=sub("gradf_I.npz"), grad_phi=sub("grad_phi_I.npz"),
                        logpdf=float(open(os.path.join(src, "logpdf_I.txt")).read()))
    np.savez_compressed(os.path.join(HERE, "infer_P.npz"), idx=idx, **meta,
                        data_e=L("data_e_field_P.npz"), data_b=L("data_b_field_P.npz"),
                        cn_ee=L("cn_ee_P.npz"), cn_bb=L("cn_bb_P.npz"), cf_ee=L("cf_ee_P.npz"), cf_bb=L("cf_bb_P.npz"),
                        cphi=L("cphi_P.npz"), m_ee=L("m_ee_P.npz"), m_bb=L("m_bb_P.npz"),
                        b_ee=L("b_ee_P.npz"), b_bb=L("b_bb_P.npz"),
                        gradf_e=sub("gradf_e_P.npz"), gradf_b=sub("gradf_b_P.npz"), grad_phi=sub("grad_phi_t_P.npz"),
                        logpdf=float(open(os.path.join(src, "logpdf_P.txt")).read()))
    # mixed parametrisation: mixing diagonals D, G in full, mixed phi gradients subsampled
    np.savez_compressed(os.path.join(HERE, "mix.npz"), idx=idx, **meta,
                        d_t=L("d_I.npz"), g=L("g_I.npz"), d_ee=L("d_ee_P.npz"), d_bb=L("d_bb_P.npz"),
                        nphi_t=L("nphi_I.npz"), nphi_p=L("nphi_P.npz"),
                        mixed_grad_phi_I=sub("mixed_grad_phi_I.npz"), mixed_grad_phi_P=sub("mixed_grad_phi_P.npz"))
    for f in sorted(os.listdir(HERE)):
        if f.endswith(".npz"):
            print(f, os.path.getsize(os.path.join(HERE, f)))


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py <reference checkout>/tests/ground_truth_data")
    main(sys.argv[1])
