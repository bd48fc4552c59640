import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "rt-nurbs_b200")):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def oracle_mod():
    import oracle

    oracle.build()
    return oracle


def load_golden(name):
    import numpy as np

    return dict(np.load(os.path.join(GOLDEN, f"{name}.npz")))


def golden_surfaces(g):
    from nrt.scenes import Surface

    out = []
    for k in range(int(g["n_surfaces"])):
        n, m, p, q = (int(x) for x in g[f"surf{k}_nmpq"])
        out.append(Surface(g[f"surf{k}_cp"], g[f"surf{k}_U"], g[f"surf{k}_V"], n, m, p, q))
    return out


def golden_rays(g):
    import oracle

    return oracle.Rays(*[g["ray_" + k] for k in ("ox", "oy", "oz", "dx", "dy", "dz")])
