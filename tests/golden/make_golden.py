"""Generate tests/golden/oracle_golden.json from the CPU FP64 oracle.

The oracle is pinned to every number the reference publishes (README.md
tables, see tests/test_oracle_pins.py); these fixtures freeze its outputs on
small, fast cases so the GPU parity tests and the CPU suite share one set of
expected values.  Run:  python tests/golden/make_golden.py
"""
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from oracle import pyoracle as po  # noqa: E402

H = dict(kappa=1.2, theta=0.05, sigma=0.35, rho=-0.4, r=0.1, T=0.6, S0=60.0, V0=0.1)


def main():
    po.build()
    cases = []
    # every option type on the reference discretization (Pricer defaults)
    spec = [(8, 0.0), (9, 0.0), (2, 50.0), (3, 50.0), (0, 50.0), (1, 50.0),
            (6, 75.0), (7, 75.0), (4, 75.0), (5, 75.0)]
    for ot, B in spec:
        for n in (8, 12):
            args = dict(H, K=[50.0, 60.0, 70.0], barrier=B, option_type=ot, n_s=n, n_v=n,
                        s_max=150.0)
            p = po.pricer_price(**args, opt=po.options(num_insert=50))
            cases.append({"args": args, "options": {"num_insert": 50}, "prices": p.tolist()})
    # other Heston parameters, ComputePipeline defaults (r 0.05, T 0.5, S0 100)
    rng = np.random.default_rng(7)
    for k in range(6):
        args = dict(kappa=float(rng.uniform(0.5, 3)), theta=float(rng.uniform(0.02, 0.15)),
                    sigma=float(rng.uniform(0.1, 0.8)), rho=float(rng.uniform(-0.9, 0)),
                    r=float(rng.uniform(0, 0.05)), T=float(rng.uniform(0.1, 2)), S0=100.0,
                    V0=float(rng.uniform(0.02, 0.2)), K=[90.0, 100.0, 110.0], barrier=0.0,
                    option_type=int(8 + k % 2), n_s=10, n_v=10)
        p = po.pricer_price(**args, opt=po.options(num_insert=50))
        cases.append({"args": args, "options": {"num_insert": 50}, "prices": p.tolist()})
    # config discretization, tight tolerances (single contracts on small grids)
    for k in range(4):
        args = dict(kappa=float(rng.uniform(0.5, 3)), theta=float(rng.uniform(0.02, 0.15)),
                    sigma=float(rng.uniform(0.1, 0.8)), rho=float(rng.uniform(-0.9, 0)),
                    r=float(rng.uniform(0, 0.05)), T=float(rng.uniform(0.1, 1.0)), S0=100.0,
                    V0=float(rng.uniform(0.02, 0.2)), K=[float(100 * rng.uniform(0.8, 1.2))],
                    barrier=0.0, option_type=int(8 + k % 2), n_s=16, n_v=12, s_max=300.0)
        o = {"disc": 1, "rtol": 1e-6, "atol": 1e-8}
        p = po.pricer_price(**args, opt=po.options(**o))
        cases.append({"args": args, "options": o, "prices": p.tolist()})
    # one-shot price + Greeks (PricingEngine), small grid
    args = dict(H, K=[55.0, 65.0], barrier=0.0, option_type=8, n_s=8, n_v=8, s_max=150.0)
    p, d, g, v, _ = po.engine_price(**args)
    engine = {"args": args, "prices": p.tolist(), "deltas": d.tolist(), "gammas": g.tolist(),
              "vegas": v.tolist()}
    # stepwise pipeline intermediates (compute_pipeline.mojo defaults, num_insert 50)
    pipe = po.Pipeline(**H, n_s=8, n_v=8, option_type=9, opt=po.options(num_insert=50))
    stepwise = {"kwargs": dict(H, n_s=8, n_v=8, option_type=9, num_insert=50),
                "s_knots": pipe.array("s_knots").tolist(), "v_knots": pipe.array("v_knots").tolist(),
                "q0": pipe.array("q0").tolist(), "qT": pipe.array("qT").tolist(),
                "dims": pipe.dims(), "price_100": pipe.price_at([100.0]).tolist()}
    out = {"generator": "tests/golden/make_golden.py", "small_cases": cases, "engine": engine,
           "stepwise": stepwise}
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "oracle_golden.json")
    with open(path, "w") as f:
        json.dump(out, f, indent=1)
    print("wrote", path, len(cases), "cases")


if __name__ == "__main__":
    main()
