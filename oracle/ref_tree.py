"""Where the genefer source tree lies (test infrastructure only).

The tree is named by the environment variable GENEFER_REF; without it, the
default that oracle/Makefile holds (its `print-ref` target) applies.  Returns
None when no tree is there, as on a machine that only runs prebuilt files.
"""
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))


def genefer_tree():
    path = os.environ.get("GENEFER_REF")
    if not path:
        try:
            r = subprocess.run(["make", "-s", "-C", HERE, "print-ref"], capture_output=True, text=True, timeout=60)
            path = r.stdout.strip() if r.returncode == 0 else ""
        except (OSError, subprocess.SubprocessError):
            path = ""
    return path if path and os.path.isdir(os.path.join(path, "src")) else None
