"""Extract known-answer values from the reference's published slurm logs.

The reference (mumairsadiq/exafmm-rd, variant ``3dpp``) has no golden vectors in
code; its only recorded outputs are the slurm logs under ``3dpp/exp/``.  Every
run there is deterministic (glibc ``drand48`` seeded with 5, fixed flags), so
the printed energies and relative L2 errors are known-answer values for the
FMM pass.  This script parses each run block (the ``input parameters=[...]``
dump printed by ``Argument::show``, ``3dpp/src/argument.cpp:72-100``) and the
comparison lines printed by ``BodyCompareResult::show``
(``3dpp/src/body.cpp:192-205``) and writes ``log_kats.json`` beside itself.

Run once, in a container where the reference tree is mounted:

    python tests/golden/extract_log_kats.py /path/to/reference
"""
import json
import os
import re
import sys

PARAM_RE = re.compile(r"^\s+(\S[^=]*?)\s+=\s+(\S+)\s*$")
CMP_RE = re.compile(r"^-+(\w+) vs (\w+)-+\[(\d+)\]")
L2_RE = re.compile(r"L2  \(p\)\s*:\s*(\S+)\s+L2  \(f\)\s*:\s*(\S+)\s+L2  \(e\)\s*:\s*(\S+)")
E_RE = re.compile(r"p-energy([12]) : (\S+)")
T_RE = re.compile(r"\[(\w+) time measured : (\S+) seconds\.\]")


def parse_log(path):
    runs = []
    cur = None
    cmp = None
    in_params = False
    with open(path, errors="replace") as f:
        for line in f:
            if line.startswith("<rtfmm_3dpp_test_pbc>") or line.startswith("rtfmm_3dp_test_fmm"):
                cur = {"log": os.path.basename(path),
                       "driver": "test_pbc" if "pbc" in line else "test_fmm",
                       "params": {}, "timers": {}, "compare": []}
                runs.append(cur)
                continue
            if cur is None:
                continue
            if line.startswith("input parameters=["):
                in_params = True
                continue
            if in_params:
                if line.startswith("]"):
                    in_params = False
                    continue
                m = PARAM_RE.match(line)
                if m:
                    cur["params"][m.group(1).strip()] = m.group(2)
                continue
            m = T_RE.search(line)
            if m:
                cur["timers"].setdefault(m.group(1), float(m.group(2)))
                continue
            m = CMP_RE.match(line)
            if m:
                cmp = {"a": m.group(1), "b": m.group(2), "n": int(m.group(3))}
                cur["compare"].append(cmp)
                continue
            if cmp is not None:
                m = L2_RE.search(line)
                if m:
                    cmp["l2p"], cmp["l2f"], cmp["l2e"] = map(float, m.groups())
                    continue
                m = E_RE.search(line)
                if m:
                    cmp["energy%s" % m.group(1)] = float(m.group(2))
    return runs


KEYS = ("P", "n", "ncrit", "images", "cycle", "seed", "dipole_correction",
        "zero_netcharge", "divide_4pi", "setting_t")


def dedupe(runs):
    """One entry per distinct (driver, parameters, comparison) with the values
    every log agrees on; runs whose energies disagree are kept apart."""
    table = {}
    for r in runs:
        p = r["params"]
        for c in r["compare"]:
            if c["a"] != "FMM" or "energy1" not in c:
                continue
            key = (r["driver"],) + tuple(p.get(k) for k in KEYS) + (c["b"], repr(c["energy1"]))
            e = table.get(key)
            if e is None:
                e = table[key] = {
                    "driver": r["driver"],
                    "params": {k: p.get(k) for k in KEYS},
                    "versus": c["b"], "energy_fmm": c["energy1"],
                    "energy_ref": c.get("energy2"), "l2p": c.get("l2p"),
                    "l2f": c.get("l2f"), "l2e": c.get("l2e"),
                    "logs": [], "fmm_kernels_s": []}
            e["logs"].append(r["log"])
            if "FMM_kernels" in r["timers"]:
                e["fmm_kernels_s"].append(r["timers"]["FMM_kernels"])
    out = []
    for e in table.values():
        e["n_runs"] = len(e["logs"])
        e["logs"] = sorted(set(e["logs"]))
        t = e.pop("fmm_kernels_s")
        e["fmm_kernels_s_mean"] = sum(t) / len(t) if t else None
        out.append(e)
    out.sort(key=lambda e: (e["driver"], int(e["params"]["P"]), int(e["params"]["images"] or 0)))
    return out


def main():
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("RTFMM_REFERENCE", "/root/reference")
    expdir = os.path.join(ref, "3dpp", "exp")
    runs = []
    for name in sorted(os.listdir(expdir)):
        if name.startswith("slurm-") and name.endswith(".out"):
            runs.extend(parse_log(os.path.join(expdir, name)))
    table = dedupe(runs)
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "log_kats.json")
    with open(out, "w") as f:
        json.dump(table, f, indent=1)
    print("wrote %d known-answer entries from %d runs to %s" % (len(table), len(runs), out))


if __name__ == "__main__":
    main()
