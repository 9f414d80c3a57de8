"""Stores micm's flow-tube regression results as a fixture.

micm's regression test (test/regression/regression_policy.hpp, TestFlowTube;
test/regression/test_regression.cpp) solves a 4-species wall-loss mechanism
with the 2-stage Rosenbrock solver and with Backward Euler for 3,600
one-second steps and keeps the concentrations in
test/regression/expected_results/{rosenbrock,backward_euler}_wall_loss.csv
(6 significant digits).  This script reads those files and writes
tests/golden/{rosenbrock,backward_euler}_wall_loss.npz.  Run from the repository root:

    python tests/golden/make_flow_tube.py [reference_root]
"""
import csv
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def main():
    if len(sys.argv) < 2:
        sys.exit(f"usage: python {os.path.basename(__file__)} <micm source tree>")
    ref = sys.argv[1]
    for solver in ("rosenbrock", "backward_euler"):
        path = os.path.join(ref, "test", "regression", "expected_results", f"{solver}_wall_loss.csv")
        with open(path) as f:
            rows = list(csv.reader(f))
        header = rows[0]
        data = np.array([[float(v) for v in r] for r in rows[1:]])
        np.savez_compressed(os.path.join(HERE, f"{solver}_wall_loss.npz"), species=np.array(header[1:]),
                            time=data[:, 0], concentrations=data[:, 1:])
        print(solver, header, data.shape)


if __name__ == "__main__":
    main()
