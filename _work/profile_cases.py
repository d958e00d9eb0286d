"""Small, self-contained cases for profiling single kernels (ncu captures of a few launches).

    python ae-engine_b200/profile_cases.py snow-clamp [iterations]

snow-clamp: the snow-collision scene (1 048 576 Stomakhin snow particles, 128^3) with every
particle's deformation gradient set to R diag(1.05, 1, 0.95) R^T for a random rotation R, so every
singular-value set lies outside the clamp band [1 - 2.5e-2, 1 + 7.5e-3] and the whole scene goes
through the snow clamp kernel (SVD return mapping) on the first substep.  Each iteration uploads
that state and runs one eager substep with stage events, printing the per-stage device times.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

import ae_mpm as M  # noqa: E402
import ae_mpm_scenes as S  # noqa: E402


def snow_clamp(iterations: int = 3) -> None:
    ctx = M.Context(0)
    sc, p = S.config2_snow()
    rng = np.random.default_rng(5)
    q, r = np.linalg.qr(rng.normal(size=(p.n, 3, 3)))
    q = q * np.sign(np.einsum("nii->ni", r))[:, None, :]
    q[np.linalg.det(q) < 0] *= -1
    p.F[:] = (q @ np.diag([1.05, 1.0, 0.95]) @ np.transpose(q, (0, 2, 1))).reshape(p.n, 9).astype(np.float32)
    w = M.World(ctx, [sc], M.exec_opts(p2g_variant=M.P2G_LANES, block_threads=128, sort_interval=16, use_graph=0))
    for it in range(iterations):
        w.upload(0, p)  # every F outside the band: the whole scene is queued for the clamp
        st = w.stage_times(1)
        print("substep", it, {k: round(v, 2) for k, v in st.items()}, flush=True)
    w.close()
    ctx.close()


CASES = {"snow-clamp": snow_clamp}

if __name__ == "__main__":
    if len(sys.argv) < 2 or sys.argv[1] not in CASES:
        sys.exit("usage: profile_cases.py {%s} [iterations]" % ",".join(CASES))
    CASES[sys.argv[1]](int(sys.argv[2]) if len(sys.argv) > 2 else 3)
