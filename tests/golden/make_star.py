"""Golden set of the star join: what the reference itself writes for tests/star_cases.py.

Builds nothing itself: it runs oracle/_ref/alenka_ref (the reference's front end,
operators and codec built for the CPU by oracle/build_ref.sh) over tables written by
oracle/refdata.py. Per dataset it runs the setup script (the CREATE INDEX statements) and
records the digest of every index file written; per case it records the script and what
the reference stored (the file when small, else its digest), or the error it stopped
with. tests/test_star.py checks the oracle (CPU) and the engine (GPU) against this.

    python tests/golden/make_star.py
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
from tests import star_cases  # noqa: E402
from tests.golden.make_ref_ops import data_digest  # noqa: E402

REF = os.path.join(ROOT, "oracle", "_ref", "alenka_ref")
OUT = os.path.join(HERE, "star")
INLINE_LIMIT = 64 * 1024


def run(d, script):
    p = os.path.join(d, "golden.sql")
    with open(p, "w") as f:
        f.write(script)
    r = subprocess.run([REF, "golden.sql"], cwd=d, capture_output=True, text=True, timeout=600)
    return r.returncode, r.stdout + r.stderr


def main():
    if not os.path.exists(REF):
        sys.exit("oracle/_ref/alenka_ref is missing: run oracle/build_ref.sh first")
    os.makedirs(OUT, exist_ok=True)
    manifest = {"reference": "oracle/_ref/alenka_ref (reference sources, Thrust OpenMP backend)",
                "datasets": star_cases.DATASETS, "setup": star_cases.SETUP, "indexes": {}, "cases": []}
    for ds_name, ds in star_cases.DATASETS.items():
        d = tempfile.mkdtemp(prefix="star_" + ds_name + "_")
        try:
            star_cases.make_dataset(d, ds, refdata)
            digest = data_digest(d)
            rc, log = run(d, star_cases.SETUP[ds_name])
            if rc != 0:
                raise RuntimeError(f"setup of {ds_name} failed: {log[-500:]}")
            manifest["indexes"][ds_name] = {
                "data_sha256": digest,
                "files": {f: hashlib.sha256(open(os.path.join(d, f), "rb").read()).hexdigest()
                          for f in star_cases.INDEX_FILES[ds_name]}}
            for c in [c for c in star_cases.CASES if c["dataset"] == ds_name]:
                fo = os.path.join(d, c["out"])
                if os.path.exists(fo):
                    os.remove(fo)
                rc, log = run(d, c["script"])
                entry = {"name": c["name"], "dataset": ds_name, "script": c["script"], "out": c["out"]}
                lines = [ln for ln in log.splitlines() if ln.startswith("(Fatal)") or ln.startswith("Required bitmap")]
                if lines or not os.path.exists(fo):
                    entry["error"] = lines[0].replace("(Fatal) ", "") if lines else f"no output (rc {rc})"
                else:
                    got = open(fo, "rb").read()
                    if len(got) <= INLINE_LIMIT:
                        fn = c["name"] + ".out"
                        with open(os.path.join(OUT, fn), "wb") as f:
                            f.write(got)
                        entry["file"] = fn
                    else:
                        entry["sha256"] = hashlib.sha256(got).hexdigest()
                        entry["lines"] = got.count(b"\n")
                manifest["cases"].append(entry)
                print(c["name"], entry.get("error", f"{entry.get('lines', '')} ok"), flush=True)
        finally:
            shutil.rmtree(d, ignore_errors=True)
    with open(os.path.join(OUT, "manifest.json"), "w") as f:
        json.dump(manifest, f, indent=1, sort_keys=True)
        f.write("\n")


if __name__ == "__main__":
    main()
