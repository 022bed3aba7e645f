"""Extract the golden values hard-coded in the reference's own tests into a JSON fixture.

Run where the reference tree is present (it is read as text; nothing of the reference
runs):  python tests/golden/extract_reference_golden.py /path/to/PSSFSS.jl
Writes tests/golden/reference_golden.json next to this script.  Every entry records the
test file and line range it came from.
"""
import json
import os
import re
import sys

NUM = r"[-+]?\d+\.\d+(?:e[-+]?\d+)?"
CPLX = re.compile(rf"({NUM})\s*([-+])\s*({NUM})im")


def cplx_on(lines, lo, hi):
    """All Julia complex literals on 1-based lines lo..hi, in order, as [re, im]."""
    out = []
    for ln in lines[lo - 1:hi]:
        for m in CPLX.finditer(ln):
            re_, sign, im = m.groups()
            out.append([float(re_), float(im) * (1 if sign == "+" else -1)])
    return out


def main(ref):
    def read(name):
        with open(os.path.join(ref, "test", name), encoding="utf-8") as f:
            return f.read().splitlines()

    fz, pgf, rwg = read("FillZY_test.jl"), read("PGF_test.jl"), read("RWGData_test.jl")
    gold = {
        "fillz": {"source": "test/FillZY_test.jl:45-46", "index_1based": [[20, 30], [100, 100]],
                  "values": cplx_on(fz, 45, 46), "tol_abs": [0.005, 0.01]},
        "filly": {"source": "test/FillZY_test.jl:77-78", "index_1based": [[20, 30], [100, 100]],
                  "values": cplx_on(fz, 77, 78), "tol_abs": [0.0001, 0.0001]},
        # [Σ1, Σ2] for u = ufact * max|β| at each ufact, checked as in test/PGF_test.jl:71-83
        "modal_series_electric": {"source": "test/PGF_test.jl:40-44", "ufact": [0.1, 0.9],
                                  "values": cplx_on(pgf, 40, 44)},
        "modal_series_magnetic": {"source": "test/PGF_test.jl:56-60", "ufact": [0.1, 0.9],
                                  "values": cplx_on(pgf, 56, 60)},
        "rwgbfft_mm": {"source": "test/RWGData_test.jl:46-48", "k": [0.0, 0.0], "psi": [0.0, 0.0],
                       "values": cplx_on(rwg, 46, 48)},  # ft[1..3], 2 components each
        "rwgbfft_inch": {"source": "test/RWGData_test.jl:56-58", "k": [20.0, -30.3], "psi": [0.8, -0.7],
                         "values": cplx_on(rwg, 56, 58)},
    }
    # mode counts per layer after choose_layer_modes! (test/Modes_test.jl, three testsets)
    md = read("Modes_test.jl")
    counts = []
    for i, ln in enumerate(md, 1):
        m = re.search(r"@test \[length\(l\.P\) for l in strata if l isa Layer\] == \[([\d,\s]+)\]", ln)
        if m:
            counts.append({"line": i, "counts": [int(x) for x in m.group(1).split(",")]})
    gold["layer_mode_counts"] = {"source": "test/Modes_test.jl", "cases": counts}
    assert len(counts) == 3, counts
    # Gblocks chosen by choose_gblocks (test/GSMs_test.jl, testsets choose_gblocks1..4):
    # Gblock(first:last, j) literals of each testset's @test lines, in order
    gs = read("GSMs_test.jl")
    starts = [i for i, ln in enumerate(gs, 1) if re.search(r'@testset "choose_gblocks\d"', ln)]
    cases = []
    for k, lo in enumerate(starts):
        hi = starts[k + 1] - 1 if k + 1 < len(starts) else len(gs)
        blocks = []
        for i in range(lo, hi + 1):
            if "@test" in gs[i - 1] and "@testset" not in gs[i - 1]:
                blocks += [[int(a), int(b), int(j)] for a, b, j in
                           re.findall(r"Gblock\((\d+):(\d+),\s*(\d+)\)", gs[i - 1])]
        cases.append({"lines": [lo, hi], "gblocks": blocks})
    gold["gblocks"] = {"source": "test/GSMs_test.jl", "cases": cases}
    assert [len(c["gblocks"]) for c in cases] == [2, 2, 2, 3], cases
    for key, n in (("fillz", 2), ("filly", 2), ("modal_series_electric", 4), ("modal_series_magnetic", 4),
                   ("rwgbfft_mm", 6), ("rwgbfft_inch", 6)):
        assert len(gold[key]["values"]) == n, (key, gold[key]["values"])
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_golden.json")
    with open(out, "w") as f:
        json.dump(gold, f, indent=1)
    print("wrote", out)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: extract_reference_golden.py <checkout of PSSFSS.jl v0.1.4>")
    main(sys.argv[1])
