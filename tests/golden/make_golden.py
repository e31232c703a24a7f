"""Generate the golden fixtures of tests/golden/ from the reference's own source text.

The reference (BCN-4He-DFT, Fortran) ships no tests; its known answers live in source:

* the Bickley finite-difference table (BLOCK DATA A(25792)): the 13-point rows for the first and
  second derivative, Dynamics_TDDFT/mates.f:786-879 (the linked copy) and the identical
  Dynamics_TDDFT/blockds.f:615-708;
* the list of admissible grid sizes, Dynamics_TDDFT/tstgrid.f90:9-13;
* functional constants (Dynamics_TDDFT/modules.f90:141-151, :229-234; He_statics/modules.f90:130)
  used by the known-answer checks b = bforce(...) ~ b4 and mu(rho0) ~ Chempo.

The table values are read as text (never compiled or run), expanded to the full 13x13 matrices the
way newder.f:99-130 does (ICON=1: the first (M*M+1)/2 entries are stored, the rest follow by the
parity sign (-1)**K), and written with their exact binary64 value as hex.

Usage:  python tests/golden/make_golden.py <path to the reference checkout>
"""
import json
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def parse_block_data(path):
    """Return {index: decimal string} for every A(I) entry of the DATA statements."""
    text = open(path, encoding="latin-1").read().splitlines()
    vals = {}
    i = 0
    head = re.compile(r"^\s+DATA \(A\(I\),I=\s*(\d+),\s*(\d+)\)/")
    num = re.compile(r"[-+]?\d+\.\d+D[-+]\d+")
    while i < len(text):
        m = head.match(text[i])
        if not m:
            i += 1
            continue
        lo, hi = int(m.group(1)), int(m.group(2))
        nums = []
        i += 1
        while len(nums) < hi - lo + 1 and i < len(text):
            nums.extend(num.findall(text[i]))
            i += 1
        for k, s in enumerate(nums[: hi - lo + 1]):
            vals[lo + k] = s
    return vals


def full_matrix(vals, m, k):
    """Expand the stored half of the (m x m) K-th derivative matrix (newder.f:99-130)."""
    ji = 1
    for i in range(3, m - 1, 2):
        ji += (i * i + 1) * (i - 2) // 2 + i
    m2 = m * m
    m21o2 = (m2 + 1) // 2
    ji += m21o2 * (k - 1)
    sig = 1.0 - 2.0 * (k % 2)
    dkf = [None] * m2
    l = ji - 1
    for j in range(1, m21o2):
        l += 1
        dkf[j - 1] = (vals[l], 1.0)
        dkf[m2 - j] = (vals[l], sig)
    l += 1
    dkf[m21o2 - 1] = (vals[l], 1.0)
    out = []
    for s, sgn in dkf:
        v = float(s.replace("D", "E")) * sgn
        out.append({"text": s, "sign": sgn, "hex": v.hex()})
    return out


def tstgrid_sizes(path):
    src = open(path, encoding="latin-1").read()
    body = src[src.index("nvalid=(/") + len("nvalid=(/"): src.index("/)")]
    return [int(t) for t in re.findall(r"\d+", body)]


def main():
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py <path to the reference checkout>")
    ref = sys.argv[1]
    dyn = os.path.join(ref, "Dynamics_TDDFT")
    linked = parse_block_data(os.path.join(dyn, "mates.f"))
    copy = parse_block_data(os.path.join(dyn, "blockds.f"))
    out = {"source": "Dynamics_TDDFT/mates.f:786-879 (== blockds.f:615-708), newder.f:99-130"}
    for k in (1, 2):
        a = full_matrix(linked, 13, k)
        b = full_matrix(copy, 13, k)
        assert [x["hex"] for x in a] == [x["hex"] for x in b], "mates.f and blockds.f differ"
        out[f"K{k}"] = a
    json.dump(out, open(os.path.join(HERE, "bickley13.json"), "w"), indent=1)

    consts = {
        "source": {
            "tstgrid": "Dynamics_TDDFT/tstgrid.f90:9-13",
            "functional": "Dynamics_TDDFT/modules.f90:141-151,229-234; He_statics/modules.f90:130",
            "bforce": "Dynamics_TDDFT/fforma.f90:256-280",
            "eos": "He_statics/rhoasin0.f90:53-63 (df = b4 rho + 3/2 cp4 rho^2 + 4/3 cpp4 rho^3)",
        },
        "tstgrid": tstgrid_sizes(os.path.join(dyn, "tstgrid.f90")),
        "eps4": 10.22, "sigma4": 2.556, "h4ot": 2.190323, "h4op": 2.359665, "b4": -718.99,
        "cp4": -2.41186e4, "cpp4": 1.85850e6, "h2o2m4": 6.05969638298,
        "densat4": 0.02184, "chempo": -7.15,
        "C": 3.1577504e4, "beta": 40.0, "den_m": 0.37,
        "mp_u": 0.02061484, "ktops": 7.63822291,
    }
    json.dump(consts, open(os.path.join(HERE, "constants.json"), "w"), indent=1)
    print("wrote bickley13.json, constants.json")


if __name__ == "__main__":
    main()
