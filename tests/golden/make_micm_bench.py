"""Writes the fixtures of micm_bench's mechanisms (TS1, Chapman) from micm itself.

Compiles tests/golden/micm_bench_dump.cpp against the reference's own headers
and its benchmark mechanisms (test/benchmark/ts1_mechanism.hpp,
test/benchmark/chapman_mechanism.hpp), runs it for each mechanism, and splits
its output into

  tests/golden/<name>_mechanism.json  the mechanism in this repository's JSON
                                      description, micm_bench's initial state
                                      and micm's state columns;
  tests/golden/<name>_micm.npz        micm's rate constants and 10 Solve(30 s)
                                      results on a 4-cell state.

The binary goes to oracle/_ref/ (reference build outputs, not committed).
Run from the repository root with the reference tree present:

    python tests/golden/make_micm_bench.py [reference_root]
"""
import json
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))


def write(name, doc):
    golden = doc.pop("golden")
    with open(os.path.join(HERE, f"{name}_mechanism.json"), "w") as f:
        json.dump(doc, f, separators=(",", ":"))
        f.write("\n")
    solves = golden["solves"]
    np.savez_compressed(
        os.path.join(HERE, f"{name}_micm.npz"),
        dt=golden["dt"], tableau=golden["tableau"], temperature=np.array(golden["temperature"]),
        pressure=np.array(golden["pressure"]), air_density=np.array(golden["air_density"]),
        initial_variables=np.array(golden["initial_variables"]),          # micm state columns
        custom_parameters=np.array(golden["custom_parameters"]),          # micm parameter columns
        rate_constants=np.array(golden["rate_constants"]),                # micm rate columns
        variables=np.array([s["variables"] for s in solves]),            # [solve][cell][micm column]
        stats=np.array([[s[k] for k in ("accepted", "rejected", "number_of_steps", "function_calls",
                                         "jacobian_updates", "decompositions", "solves")] for s in solves]),
        converged=np.array([s["state"] == "Converged" for s in solves]))
    for f in (f"{name}_mechanism.json", f"{name}_micm.npz"):
        print(f, os.path.getsize(os.path.join(HERE, f)), "bytes")


def main():
    if len(sys.argv) < 2:
        sys.exit(f"usage: python {os.path.basename(__file__)} <micm source tree>")
    ref = sys.argv[1]
    out_dir = os.path.join(ROOT, "oracle", "_ref")
    os.makedirs(out_dir, exist_ok=True)
    exe = os.path.join(out_dir, "micm_bench_dump")
    subprocess.run(["g++", "-std=c++20", "-O1", "-ffp-contract=off", "-DMICM_DEFAULT_VECTOR_SIZE=4",
                    "-I" + os.path.join(ref, "include"), "-I" + os.path.join(ref, "test", "benchmark"),
                    "-o", exe, os.path.join(HERE, "micm_bench_dump.cpp")], check=True)
    for name in ("ts1", "chapman"):
        write(name, json.loads(subprocess.run([exe, name], check=True, capture_output=True, text=True).stdout))


if __name__ == "__main__":
    main()
