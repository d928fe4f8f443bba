"""Runs the SPAMMM reference's own tests of the probe-particle AFM path against
this drop-in and writes the pass/fail list.

    python tests/refsuite/run_reference_suite.py --ref PATH [--gpu] [--out FILE]

PATH (or $SPAMMM_REF) is the root of the reference tree; its test files run
unmodified, in place: tests/SPM/test_scan_contract.py, test_texel_centers.py
and test_afm_morse.py.  The plugin spm_reference_alias.py (next to this file)
points their imports of spammm.SPM.AFM / AFM_utils at spammm_b200 and supplies
stand-ins for pyopencl (grid read-back only) and matplotlib.  Without --gpu the
tests not marked gpu run (no CUDA needed); with --gpu the gpu-marked ones.
Nothing is written into the reference tree (no bytecode, no pytest cache; the
tests' debug output goes to a temporary working directory).
"""
import argparse
import os
import subprocess
import sys
import tempfile
import xml.etree.ElementTree as ET

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
FILES = ("tests/SPM/test_scan_contract.py", "tests/SPM/test_texel_centers.py", "tests/SPM/test_afm_morse.py")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("SPAMMM_REF"))
    ap.add_argument("--gpu", action="store_true")
    ap.add_argument("--out", default=None)
    args = ap.parse_args()
    if not args.ref:
        ap.error("give the reference tree with --ref PATH or SPAMMM_REF")
    ref = os.path.abspath(args.ref)
    work = tempfile.mkdtemp(prefix="spm_refsuite_")
    xml = os.path.join(work, "junit.xml")
    env = dict(os.environ, PYTHONDONTWRITEBYTECODE="1",
               PYTHONPATH=os.pathsep.join([HERE, ROOT, ref, os.environ.get("PYTHONPATH", "")]))
    cmd = [sys.executable, "-m", "pytest", *[os.path.join(ref, f) for f in FILES], "-p", "spm_reference_alias",
           "-p", "no:cacheprovider", "--rootdir", ref, "-q", "-rA", f"--junitxml={xml}",
           "-m", "gpu" if args.gpu else "not gpu", "-o", "addopts="]
    proc = subprocess.run(cmd, cwd=work, env=env, capture_output=True, text=True)
    rows = []
    if os.path.exists(xml):
        for tc in ET.parse(xml).getroot().iter("testcase"):
            name = f"{tc.get('classname', '').split('.')[-1]}::{tc.get('name')}"
            status, msg = "passed", ""
            for tag in ("failure", "error", "skipped"):
                el = tc.find(tag)
                if el is not None:
                    status = {"failure": "failed", "error": "error", "skipped": "skipped"}[tag]
                    msg = (el.get("message") or "").splitlines()[0][:160] if el.get("message") else ""
            rows.append((name, status, msg))
    lines = [f"# reference tests against the drop-in ({'gpu' if args.gpu else 'not gpu'} subset)", "",
             "Command: `python tests/refsuite/run_reference_suite.py --ref <reference root>"
             + (" --gpu" if args.gpu else "") + "`", "",
             "| test | result | note |", "|---|---|---|"]
    lines += [f"| {n} | {s} | {m.replace('|', '/')} |" for n, s, m in rows]
    counts = {s: sum(1 for r in rows if r[1] == s) for s in ("passed", "failed", "error", "skipped")}
    lines += ["", "Totals: " + ", ".join(f"{k} {v}" for k, v in counts.items()), ""]
    text = "\n".join(lines)
    if args.out:
        with open(args.out, "w") as f:
            f.write(text)
    print(text)
    if proc.returncode not in (0, 1):
        print(proc.stdout[-4000:], proc.stderr[-4000:])
    return 0 if counts["failed"] == 0 and counts["error"] == 0 else 1


if __name__ == "__main__":
    sys.exit(main())
