"""Generate tests/golden/regression_sums.json from the reference's own
regression data (examples/*/regression_data/frameNNNN.txt: per-field sums of
q over interior cells, as check_frame compares them).

Run in a checkout that has the reference at REFERENCE (default
/root/reference); the JSON it writes is committed so the tests need no
reference tree at run time.
"""
import json
import os
import sys

REFERENCE = os.environ.get("REFERENCE", "/root/reference")
CASES = {
    # example directory: (test file with the overrides, fields checked)
    "acoustics_1d_example1": "examples/acoustics_1d_example1/test_acoustics_1d_example1.py",
    "acoustics_1d_heterogeneous": "examples/acoustics_1d_heterogeneous/test_acoustics_1d_heterogeneous.py",
    "acoustics_3d_heterogeneous": "examples/acoustics_3d_heterogeneous/test_acoustics_3d_heterogeneous.py",
    "advection_2d_annulus": "examples/advection_2d_annulus/test_advection_2d_annulus.py",
}


def main(out=os.path.join(os.path.dirname(os.path.abspath(__file__)), "regression_sums.json")):
    golden = {}
    for name, test in CASES.items():
        d = os.path.join(REFERENCE, "examples", name, "regression_data")
        frames = {}
        for fn in sorted(os.listdir(d)):
            if fn.startswith("frame") and fn.endswith(".txt"):
                with open(os.path.join(d, fn)) as f:
                    frames[int(fn[5:9])] = [float(x) for x in f.read().split()]
        golden[name] = {"source": f"examples/{name}/regression_data", "test": test,
                        "frames": frames}
    with open(out, "w") as f:
        json.dump(golden, f, indent=1, sort_keys=True)
    print(f"wrote {out}", file=sys.stderr)


if __name__ == "__main__":
    main()
