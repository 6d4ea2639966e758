"""Golden outputs of the reference's own text loader: for every case of tests/text_cases.py
the text file is written, the reference CLI (oracle/_ref/alenka_ref, its operators built
for the CPU) runs the case's scripts (LOAD ... STORE ... BINARY, then a query over the
stored table), and the SHA-256 of every
file it wrote for the stored table (segments and headers) and of its text outputs go to
tests/golden/text_load.json. tests/test_text_load.py checks the engine against them.

    python tests/golden/make_text_load.py
"""
import hashlib
import json
import os
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from tests import text_cases  # noqa: E402

REF = os.path.join(ROOT, "oracle", "_ref", "alenka_ref")


def sha(b):
    return hashlib.sha256(b).hexdigest()


def main():
    out = {}
    for name, case in sorted(text_cases.CASES.items()):
        d = tempfile.mkdtemp(prefix="textload_")
        text = case["text"]().encode()
        with open(os.path.join(d, text_cases.FILES[name]), "wb") as f:
            f.write(text)
        for k, script in enumerate(case["scripts"]):
            with open(os.path.join(d, f"s{k}.sql"), "w") as f:
                f.write(script)
            r = subprocess.run([REF, f"s{k}.sql"], cwd=d, capture_output=True, text=True, timeout=600)
            if r.returncode != 0:
                raise SystemExit(f"{name}: reference failed: {r.stdout[-400:]} {r.stderr[-400:]}")
        files = {}
        for fn in sorted(os.listdir(d)):
            if fn.startswith(case["table"] + ".") or fn == case["table"] or fn.endswith("_q.txt"):
                files[fn] = sha(open(os.path.join(d, fn), "rb").read())
        out[name] = {"text_sha256": sha(text), "files": files}
    with open(os.path.join(HERE, "text_load.json"), "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)
    print("wrote", os.path.join(HERE, "text_load.json"), {k: len(v["files"]) for k, v in out.items()})


if __name__ == "__main__":
    main()
