"""How far the reference's own 500-step Chebyshev run (run_cheb_l32m4.npz) moves
under rounding-level changes that keep its mathematics, to put the FP64 GPU
run's distance from it in scale.  Runs the reference itself (CPU, FP64,
TorchDynamo disabled), so it needs the reference checkout and is not a test:

    python tests/golden/reference_sensitivity.py [--fields] [--fold] [--ourD] [--nl EPS]

--fields  multiply every field by (1 + 1e-16 N(0,1)) after every step
--fold    apply the implicit solves in the GPU library's form: the DCT-I
          multiplied into each degree's inverse (one dense product per degree,
          grid values out) instead of the inverse followed by costf
--ourD    use this package's Chebyshev derivative matrices (magic_b200.radial:
          the same published construction, built in numpy) instead of the
          reference's own (they differ by ~4.5e-16 of their largest entry)
--nl EPS  add noise of EPS times each equation's largest explicit term to the
          explicit terms every step (the size of the FP64 stage's rounding
          differences from the reference at this l_max is ~1e-14)

Prints the largest difference of w, z, s, b, aj, p after step 500 from the
reference's unmodified run, relative to each field's largest value.  Recorded
results (this container, 8 cores): --fields: z 8.9e-14; --fold: z 4.0e-13;
--ourD: z 2.7e-13; --nl 1e-14: z 6.2e-14; --fold --ourD --nl 1e-14: z 4.6e-13;
the GPU's FP64 run: z 4.4e-12.
"""

import argparse
import os
import sys

import numpy as np

REF = "/root/reference/src"
HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--fields", action="store_true")
    ap.add_argument("--fold", action="store_true")
    ap.add_argument("--ourD", action="store_true")
    ap.add_argument("--nl", type=float, default=0.0)
    args = ap.parse_args()
    os.environ["TORCHDYNAMO_DISABLE"] = "1"
    sys.path.insert(0, REF)
    from magic_torch.config import configure

    configure({"l_max": 32, "minc": 4, "n_r_max": 33, "ek": 1e-3, "ra": 1e5, "pr": 1.0,
               "prmag": 5.0, "dtmax": 1e-4, "mode": 0, "device": "cpu", "use_shtns": False})
    import torch
    from magic_torch import blocking, dt_fields, fields, params, step_time, update_b, update_wp
    from magic_torch import radial_derivatives as rd
    from magic_torch.cosine_transform import costf
    from magic_torch.init_fields import initialize_fields

    N, lm = params.n_r_max, params.lm_max
    if args.fold:
        Cl = costf(torch.eye(N, dtype=torch.float64)).T.contiguous()  # costf(x) = Cl @ x
        Cl2 = torch.block_diag(Cl, Cl)
        build = step_time.build_all_matrices

        def build_folded(*a, **k):
            build(*a, **k)
            step_time._scalar_inv = torch.matmul(Cl, step_time._scalar_inv)
            update_wp._wp_inv_by_l = torch.matmul(Cl2, update_wp._wp_inv_by_l)
            update_b._b_inv_by_l = torch.matmul(Cl, update_b._b_inv_by_l)
            update_b._j_inv_by_l = torch.matmul(Cl, update_b._j_inv_by_l)

        step_time.build_all_matrices = build_folded
        solve_p0 = update_wp.solve_p0
        update_wp.solve_p0 = lambda rhs: Cl @ solve_p0(rhs)
        step_time.costf = lambda x: x
        update_b.costf = lambda x: x
    if args.ourD:
        sys.path.insert(0, ROOT)
        from magic_b200.radial import cheb_matrices

        _, D1n, D2n, D3n = cheb_matrices(N, 0.35)
        D1t, D2t, D3t = (torch.as_tensor(np.asarray(x)).T.contiguous() for x in (D1n, D2n, D3n))
        rd._D1_real_T, rd._D2_real_T, rd._D3_real_T = D1t, D2t, D3t
        rd._D1, rd._D2, rd._D3 = (x.T.contiguous().to(torch.complex128) for x in (D1t, D2t, D3t))
        step_time._D12_T = torch.cat([D1t, D2t], dim=1)
        step_time._D123_T = torch.cat([D1t, D2t, D3t], dim=1)
        step_time._D1_cd, step_time._D2_cd, step_time._D3_cd = rd._D1, rd._D2, rd._D3
        update_wp._D2_cd_wp, update_wp._D3_cd_wp = rd._D2, rd._D3
    gen = torch.Generator().manual_seed(123)
    if args.nl > 0:
        lm_loop = step_time._fused_lm_loop_fast

        def perturbed(*a, **k):
            e = dt_fields._all_expl[:, :, 0]
            sc = e.abs().reshape(-1, lm, N).amax(dim=(1, 2)).repeat_interleave(lm)[:, None]
            e.add_(args.nl * sc * torch.complex(
                torch.randn(e.shape, generator=gen, dtype=torch.float64),
                torch.randn(e.shape, generator=gen, dtype=torch.float64)))
            return lm_loop(*a, **k)

        step_time._fused_lm_loop_fast = perturbed
    # the fixture's initial state (make_golden.py: the reference's initial fields
    # plus seeded entropy noise 1e-5 on the interior levels)
    initialize_fields()
    g = torch.Generator().manual_seed(0)
    m0 = blocking.st_lm2m == 0
    c = torch.complex(torch.randn(lm, N, generator=g, dtype=torch.float64),
                      torch.randn(lm, N, generator=g, dtype=torch.float64)) * 1e-5
    c[m0] = c[m0].real.to(c.dtype)
    fields.s_LMloc[:, 1:-1] += c[:, 1:-1]
    step_time.setup_initial_state()
    step_time.initialize_dt(1e-4)
    names = ("s_LMloc", "w_LMloc", "z_LMloc", "b_LMloc", "aj_LMloc")
    for step in range(1, 501):
        step_time.one_step(step, 1e-4)
        if args.fields:
            for k in names:
                f = getattr(fields, k)
                f.mul_(1.0 + 1e-16 * torch.randn(f.shape, generator=gen, dtype=torch.float64))
    z = np.load(os.path.join(HERE, "run_cheb_l32m4.npz"))
    for k in ("w", "z", "s", "b", "aj", "p"):
        a = getattr(fields, k + "_LMloc").numpy()
        print(k, float(np.abs(a - z["500:" + k]).max() / np.abs(z["500:" + k]).max()))


if __name__ == "__main__":
    main()
