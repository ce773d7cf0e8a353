"""Build recipe for oracle/_ref/libvfsref.so: the reference's own hot-path sources,
compiled unmodified with g++ against the single-rank PETSc/MPI shim in oracle/shim/.

Test infrastructure only.  It needs the reference checkout (REF_DIR, default the
read-only mount) and writes only under oracle/_ref/.  The library is git-ignored but
travels with the repository snapshot, so the GPU-side tests can use it without the
reference sources.

Reference functions that live in sources outside this list (turbines, FSI, wave
models ...) are never reached by the oracle driver; the link gives each of them a
stub that aborts with its name (shim_unresolved), and each global that only those
sources define gets zeroed storage.
"""
import os
import re
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
OBJ = os.path.join(OUT, "obj")
SHIM = os.path.join(HERE, "shim")
LIB = os.path.join(OUT, "libvfsref.so")
# The reference checkout: the REF_DIR environment variable, else the read-only mount.
REF_DIR = os.environ.get("REF_DIR", "/root/reference")

# Reference translation units compiled into the oracle (the hot path plus the set-up
# code it needs: grid input, metrics, BCs, IB interpolation, LES, globals in main.c;
# sediment_transport-Y.c for the wall model the IB interpolation calls,
# wall_function_roughness_a).
REF_SOURCES = [
    "main.c", "init.c", "metrics.c", "momentum.c", "rhs.c", "rhs2.c", "k-omega.c",
    "poisson.c", "poisson_hypre.c", "les.c", "bcs.c", "wallfunction.c", "ibm.c",
    "compgeom.c", "level.c", "variables.c", "sediment_transport-Y.c",
]
CXXFLAGS = ["-std=c++11", "-O2", "-fPIC", "-w", "-fpermissive", "-ffp-contract=off",
            "-DNDEBUG", "-I" + SHIM]


def _run(cmd, **kw):
    return subprocess.run(cmd, check=False, capture_output=True, text=True, **kw)


# ibm.c has non-void functions that end without a return (nearestcell1, ibm.c:1366-1512);
# g++ 13 at -O2 treats the missing return as unreachable and the generated code runs on
# past the function's end.  At -O0 the end becomes a single trap instruction, which the
# oracle driver catches (ref_driver.cpp, call_nearestcell1).  SSE2 double arithmetic is the
# same at either level.
O0_SOURCES = ("ibm.c",)


def _compile(src, obj, extra_inc):
    newest = max(os.path.getmtime(src), os.path.getmtime(os.path.abspath(__file__)),
                 max(os.path.getmtime(os.path.join(SHIM, h)) for h in os.listdir(SHIM)))
    if os.path.exists(obj) and os.path.getmtime(obj) >= newest:
        return
    flags = [("-O0" if f == "-O2" and os.path.basename(src) in O0_SOURCES else f) for f in CXXFLAGS]
    r = _run(["g++"] + flags + ["-I" + extra_inc, "-c", src, "-o", obj])
    if r.returncode != 0:
        raise RuntimeError("oracle/_ref: compile failed for %s\n%s" % (src, r.stderr[-4000:]))


def _stub_asm(func_syms, data_syms):
    lines = ["    .text"]
    for n, s in enumerate(sorted(func_syms)):
        lines += ["    .globl %s" % s, "    .type %s, @function" % s, "%s:" % s,
                  "    leaq .Lstubname%d(%%rip), %%rdi" % n, "    jmp shim_unresolved@PLT"]
    lines.append("    .section .rodata")
    for n, s in enumerate(sorted(func_syms)):
        lines += [".Lstubname%d:" % n, '    .asciz "%s"' % s]
    lines.append("    .bss")
    for s in sorted(data_syms):
        lines += ["    .globl %s" % s, "    .type %s, @object" % s, "    .align 64",
                  "%s:" % s, "    .zero 4096", "    .size %s, 4096" % s]
    lines.append('    .section .note.GNU-stack,"",@progbits')
    return "\n".join(lines) + "\n"


def build(ref_dir=None, verbose=False):
    """Compile the reference sources + shim + driver into oracle/_ref/libvfsref.so."""
    ref_dir = ref_dir or REF_DIR
    if not os.path.isdir(ref_dir):
        raise FileNotFoundError("reference sources not found at %s" % ref_dir)
    os.makedirs(OBJ, exist_ok=True)
    objs = []
    for src in REF_SOURCES:
        obj = os.path.join(OBJ, src.replace(".c", ".o").replace("-", "_"))
        _compile(os.path.join(ref_dir, src), obj, ref_dir)
        objs.append(obj)
    for src in ("shim.cpp", "ref_driver.cpp"):
        obj = os.path.join(OBJ, src.replace(".cpp", ".o"))
        _compile(os.path.join(SHIM, src), obj, ref_dir)
        objs.append(obj)

    # Undefined global-namespace C++ functions -> aborting stubs (two passes: the
    # linker then names any remaining plain symbol, which is reference data).
    partial = os.path.join(OBJ, "partial.o")
    r = _run(["ld", "-r", "-o", partial] + objs)
    if r.returncode != 0:
        raise RuntimeError("oracle/_ref: partial link failed\n" + r.stderr)
    undef = _run(["nm", "-u", partial]).stdout.split()
    funcs = {s for s in undef if re.match(r"^_Z[0-9]", s)}
    data = set()
    stub_s = os.path.join(OBJ, "stubs.s")
    stub_o = os.path.join(OBJ, "stubs.o")
    for _ in range(3):
        with open(stub_s, "w") as f:
            f.write(_stub_asm(funcs, data))
        r = _run(["gcc", "-c", stub_s, "-o", stub_o])
        if r.returncode != 0:
            raise RuntimeError("oracle/_ref: stub assembly failed\n" + r.stderr)
        r = _run(["g++", "-shared", "-o", LIB + ".tmp", "-Wl,--no-undefined"] + objs +
                 [stub_o, "-lm"])
        if r.returncode == 0:
            os.replace(LIB + ".tmp", LIB)
            if verbose:
                print("oracle/_ref: built %s (%d function stubs, %d data stubs)"
                      % (LIB, len(funcs), len(data)))
            return LIB
        missing = set(re.findall(r"undefined reference to `([^'(]+)'", r.stderr))
        if not missing:
            raise RuntimeError("oracle/_ref: link failed\n" + r.stderr[-4000:])
        data |= {m for m in missing if not m.startswith("_Z")}
        funcs |= {m for m in missing if m.startswith("_Z")}
    raise RuntimeError("oracle/_ref: link did not converge\n" + r.stderr[-4000:])


if __name__ == "__main__":
    build(sys.argv[1] if len(sys.argv) > 1 else REF_DIR, verbose=True)
