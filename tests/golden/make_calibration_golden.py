"""Extracts the reference's published PDHG per-iteration calibration
(results/gpu/calibrate.json, the output of `calibrateBandwidth`,
src/parametric/parametric.cpp:531-585, on its laptop CPU and GPU) into
calibration_published.json: per scale, the instance's rows, columns and
nonzeros and the CPU and GPU seconds per iteration and effective GB/s.

Run from the repository root, with the reference tree present:

    python tests/golden/make_calibration_golden.py
"""
import json
import os

HERE = os.path.dirname(os.path.abspath(__file__))
REF = os.environ.get("PRAMANA_REFERENCE", "/root/reference")


def main():
    with open(os.path.join(REF, "results", "gpu", "calibrate.json")) as f:
        d = json.load(f)
    out = {"gpu": d["gpu"]["name"], "cpu_threads": d["cpu_threads"], "scales": []}
    for r in d["pdhg_iteration_timing"]:
        out["scales"].append({"rows": r["rows"], "cols": r["cols"], "nnz": r["nnz"],
                              "cpu_seconds_per_iteration": r["cpu"]["seconds_per_iteration"],
                              "cpu_effective_GBs": r["cpu"]["effective_GBs"],
                              "gpu_seconds_per_iteration": r["gpu"]["seconds_per_iteration"],
                              "gpu_effective_GBs": r["gpu"]["effective_GBs"]})
    with open(os.path.join(HERE, "calibration_published.json"), "w") as f:
        json.dump(out, f, indent=1)
    print(json.dumps(out)[:300])


if __name__ == "__main__":
    main()
