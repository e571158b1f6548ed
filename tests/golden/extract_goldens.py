"""Extract the golden values of the reference's integration tests into
reference_goldens.json.

Reads the reference test files as text (no Julia needed): every
``expected_error[<form>, <level>] = <value>`` line and the entropy-drift
tolerances ``@test abs(Δη) <= <n>eps(FT)``.  Run once where the reference is
mounted:

    python tests/golden/extract_goldens.py /path/to/Atum.jl

The JSON records, for each value, the file and line it came from.
"""
import json
import os
import re
import sys

FILES = [
    "test/advection/wave_1d.jl", "test/advection/wave_2d.jl", "test/advection/wave_3d.jl",
    "test/advection/imex_wave_2d.jl", "test/advection/entropy_conservation_1d.jl",
    "test/euler/wave_1d.jl", "test/euler/wave_2d.jl", "test/euler/wave_3d.jl",
    "test/euler/isentropicvortex.jl", "test/euler/entropy_conservation_1d.jl",
    "test/shallow_water/entropy_conservation_1d.jl", "test/euler_gravity/linear.jl",
]
FORM = {"WeakForm()": "weak", "FluxDifferencingForm(EntropyConservativeFlux())": "fd_ec",
        "FluxDifferencingForm(CentralFlux())": "fd_central"}


def main(root):
    out = {}
    for rel in FILES:
        key = rel[len("test/"):-len(".jl")]
        entry = {"values": [], "entropy_tol_eps": None, "source": rel}
        with open(os.path.join(root, rel), encoding="utf-8") as f:
            for ln, line in enumerate(f, 1):
                m = re.search(r"expected_error\[(.+?), (\d+)\] = ([-+0-9.eE]+)", line)
                if m:
                    entry["values"].append({"form": FORM[m.group(1)], "level": int(m.group(2)),
                                            "value": float(m.group(3)), "line": ln})
                    continue
                m = re.search(r"expected_error\[(\d+)\] = ([-+0-9.eE]+)", line)
                if m:
                    entry["values"].append({"form": "weak", "level": int(m.group(1)),
                                            "value": float(m.group(2)), "line": ln})
                    continue
                m = re.search(r"@test abs\(Δη\) <= (\d+)eps", line)
                if m:
                    entry["entropy_tol_eps"] = int(m.group(1))
                    entry["entropy_tol_line"] = ln
        out[key] = entry
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_goldens.json")
    with open(dst, "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)
    print("wrote", dst, sum(len(v["values"]) for v in out.values()), "values")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/extract_goldens.py <path to the Atum.jl checkout>")
    main(sys.argv[1])
