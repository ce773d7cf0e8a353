"""Build recipe for oracle/liboracle.so, the C restatement of the reference's projection
path (oracle/vfs_oracle.c).  Test infrastructure; plain gcc, no FMA contraction so its
arithmetic follows the written operation order."""
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "vfs_oracle.c")
LIB = os.path.join(HERE, "liboracle.so")


def build(verbose=False):
    if os.path.exists(LIB) and os.path.getmtime(LIB) >= os.path.getmtime(SRC):
        return LIB
    cmd = ["gcc", "-O2", "-std=c11", "-fPIC", "-shared", "-ffp-contract=off", "-Wall", "-Wno-unused-variable",
           SRC, "-o", LIB + ".tmp", "-lm"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("oracle build failed\n" + r.stderr[-4000:])
    os.replace(LIB + ".tmp", LIB)
    if verbose:
        print(LIB)
    return LIB


if __name__ == "__main__":
    build(verbose=True)
