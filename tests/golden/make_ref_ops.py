"""Golden outputs of the reference's own operators.

Builds nothing itself: it runs oracle/_ref/alenka_ref (the reference's bison front end,
operators and codec built for the CPU by oracle/build_ref.sh) over seeded tables
written by oracle/refdata.py, and records for every case the script, the digest of the
input files, and what the reference stored (the file itself when small, else its
SHA-256 and line count) or the fatal error it stopped with. tests/test_ref_golden.py
checks the oracle (CPU) and the engine (GPU) against this manifest.

    python tests/golden/make_ref_ops.py                   # all cases
    python tests/golden/make_ref_ops.py --small           # cases below 1M rows only
    python tests/golden/make_ref_ops.py --only <dataset>  # one dataset's cases
The 600M-row dataset needs about 10 GB of disk and a few minutes of the reference.
"""
import hashlib
import json
import os
import shutil
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import refdata  # noqa: E402
from tests import ref_cases  # noqa: E402

REF = os.path.join(ROOT, "oracle", "_ref", "alenka_ref")
OUT = os.path.join(HERE, "ref_ops")
INLINE_LIMIT = 64 * 1024  # larger outputs are kept as a digest


def data_digest(d):
    h = hashlib.sha256()
    for f in sorted(os.listdir(d)):
        p = os.path.join(d, f)
        if not os.path.isfile(p) or f.endswith((".sql", ".txt")):
            continue
        h.update(f.encode() + b"\0")
        with open(p, "rb") as fh:
            while True:
                b = fh.read(1 << 24)
                if not b:
                    break
                h.update(b)
    return h.hexdigest()


def run_reference(d, script, out):
    p = os.path.join(d, "golden.sql")
    with open(p, "w") as f:
        f.write(script)
    fo = os.path.join(d, out)
    if os.path.exists(fo):
        os.remove(fo)
    r = subprocess.run([REF, "golden.sql"], cwd=d, capture_output=True, text=True, timeout=3600)
    fatal = [ln for ln in r.stdout.splitlines() + r.stderr.splitlines() if ln.startswith("(Fatal)")]
    if fatal:
        return None, fatal[0][len("(Fatal) "):].strip()
    if r.returncode != 0 or not os.path.exists(fo):
        raise RuntimeError(f"reference failed ({r.returncode}): {r.stdout[-500:]} {r.stderr[-500:]}")
    with open(fo, "rb") as f:
        return f.read(), None


def main():
    small = "--small" in sys.argv
    only = sys.argv[sys.argv.index("--only") + 1] if "--only" in sys.argv else None
    if not os.path.exists(REF):
        sys.exit("oracle/_ref/alenka_ref is missing: run oracle/build_ref.sh first")
    os.makedirs(OUT, exist_ok=True)
    manifest = {"reference": "oracle/_ref/alenka_ref (reference sources, Thrust OpenMP backend)", "cases": []}
    old = {}
    mpath = os.path.join(OUT, "manifest.json")
    if (small or only) and os.path.exists(mpath):
        old = {c["name"]: c for c in json.load(open(mpath))["cases"]}
    for ds_name, ds in ref_cases.DATASETS.items():
        cases = [c for c in ref_cases.CASES if c["dataset"] == ds_name]
        if (small and ds["rows"] >= 1_000_000) or (only and ds_name != only):
            manifest["cases"] += [old[c["name"]] for c in cases if c["name"] in old]
            continue
        d = tempfile.mkdtemp(prefix="golden_" + ds_name + "_")
        try:
            ref_cases.make_dataset(d, ds, refdata)
            digest = data_digest(d)
            for c in cases:
                got, err = run_reference(d, c["script"], c["out"])
                entry = {"name": c["name"], "dataset": ds_name, "script": c["script"], "out": c["out"],
                         "mode": c.get("mode", "bytes"), "data_sha256": digest}
                if "segments_skipped" in c:
                    entry["segments_skipped"] = c["segments_skipped"]
                if err is not None:
                    entry["error"] = err
                elif len(got) <= INLINE_LIMIT:
                    fn = c["name"] + ".out"
                    with open(os.path.join(OUT, fn), "wb") as f:
                        f.write(got)
                    entry["file"] = fn
                else:
                    entry["sha256"] = hashlib.sha256(got).hexdigest()
                    entry["lines"] = got.count(b"\n")
                    entry["sorted_sha256"] = hashlib.sha256(b"\n".join(sorted(got.split(b"\n")))).hexdigest()
                manifest["cases"].append(entry)
                print(c["name"], "error: " + err if err else f"{len(got)} bytes", flush=True)
        finally:
            shutil.rmtree(d, ignore_errors=True)
    manifest["datasets"] = ref_cases.DATASETS
    with open(mpath, "w") as f:
        json.dump(manifest, f, indent=1, sort_keys=True)
        f.write("\n")


if __name__ == "__main__":
    main()
