"""Build libspinsim_b200.so in-tree for sm_100a.

* Built-in field kernels (tabulated, tones) and the scan kernels are compiled to sm_100a SASS.
* Kernels for user fields are compiled to LTO-IR fatbins (one per method variant), embedded in the
  library with ``.incbin`` and linked with the user's LTO-IR by nvJitLink at plan creation.

Usage: ``python -m spinsim_b200.build [-j N] [--force]``.  Objects are rebuilt only when their
command line or any source under ``csrc/`` changed.
"""
import argparse
import concurrent.futures as cf
import hashlib
import itertools
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.environ.get("SPINSIM_BUILD_DIR", os.path.join(HERE, "_build"))
GEN = os.path.join(BUILD, "gen")
LIB = os.environ.get("SPINSIM_LIB", os.path.join(HERE, "libspinsim_b200.so"))
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

ARCH_SASS = "-gencode=arch=compute_100a,code=sm_100a"
ARCH_LTO = "-gencode=arch=compute_100a,code=lto_100a"
COMMON = ["-std=c++17", "-O3", "-lineinfo", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC",
          f"-I{CSRC}", f"-I{GEN}", f"-I{INCLUDE}"] + os.environ.get("SPINSIM_NVCC_FLAGS", "").split()

INTEG = {0: "cf4", 1: "euler", 2: "heun"}
EXPO = {0: "an", 1: "lt", 2: "lt8"}
FIELD = {0: "user", 1: "table", 2: "tones"}
PREC = {0: "f64", 1: "f32b"}


def nvcc():
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def host_cc():
    return "/usr/bin/gcc" if os.path.exists("/usr/bin/gcc") else "gcc"


def variants():
    """(dims, integ, expo_h, expo_o, prec) method variants that get kernels."""
    out = []
    for integ in (0, 1, 2):
        for eh in (0, 1):
            out.append((2, integ, eh, 1, 0))
        for eo in (1, 2):
            out.append((3, integ, 0, eo, 0))
    # Mixed-dimension batches: Magnus CF4 with either spin-half exponentiator, spin-one Lie-Trotter.
    out.append((0, 0, 0, 1, 0))
    out.append((0, 0, 1, 1, 0))
    # FP32-bulk: Magnus CF4 for single spins and mixed batches; Euler and Heun for single spins.
    for eh in (0, 1):
        out.append((2, 0, eh, 1, 1))
    out.append((3, 0, 0, 1, 1))
    out.append((0, 0, 0, 1, 1))
    out.append((0, 0, 1, 1, 1))
    for integ in (1, 2):
        for eh in (0, 1):
            out.append((2, integ, eh, 1, 1))
        out.append((3, integ, 0, 1, 1))
    return out


def vname(v, field=None):
    dims, integ, eh, eo, prec = v
    s = f"d{dims}_{INTEG[integ]}_{EXPO[eh]}_{EXPO[eo]}_{PREC[prec]}"
    return s if field is None else f"{s}_{FIELD[field]}"


def tmpl(v, field, minb=None):
    dims, integ, eh, eo, prec = v
    base = f"{dims}, {integ}, {eh}, {eo}, {field}, {prec}"
    return base if minb is None else f"{base}, {minb}"


# Register budgets built for every built-in kernel: minimum resident 128-thread CTAs per SM.
MINB = (2, 3, 4)
# Tighter budgets (96 and 80 registers) for the FP32-bulk tabulated-field kernels, the serving path,
# whose latency-bound table lookups gain from residency more than they lose to spills.
MINB_TIGHT = (5, 6)
# Register budgets of the tensor-path tone kernels (128-thread CTAs): 5 -> 102, 4 -> 128, 3 -> 168 registers.
DMMA_MINB = (3, 4, 5, 6)


def gen_sources():
    os.makedirs(GEN, exist_ok=True)
    units = []  # (kind, name, source path)
    reg_decl, builtin_rows, user_rows = [], [], []
    for v in variants():
        for field in (1, 2):
            for minb in MINB + (MINB_TIGHT if (v[4] == 1 and field == 1) else ()):
                name = f"{vname(v, field)}_b{minb}"
                src = os.path.join(GEN, f"k_{name}.cu")
                t = tmpl(v, field, minb)
                body = (f'#include "evolve_kernel.cuh"\n'
                        f"namespace spinsim {{\ntemplate __global__ void evolve_kernel<{t}>(EvolveArgs);\n}}\n"
                        f'extern "C" const void* spinsim_kget_{name}(void) {{\n'
                        f"    return (const void*)&spinsim::evolve_kernel<{t}>;\n}}\n")
                write_if_changed(src, body)
                units.append(("sass", name, src))
                reg_decl.append(f'extern "C" const void* spinsim_kget_{name}(void);')
                builtin_rows.append(f"    {{{v[0]}, {v[1]}, {v[2]}, {v[3]}, {field}, {v[4]}, {minb}, spinsim_kget_{name}}},")
        name = vname(v)
        src = os.path.join(GEN, f"u_{name}.cu")
        body = ("#define SPINSIM_USER_FIELD 1\n"
                '#include "evolve_kernel.cuh"\n'
                f'extern "C" __global__ void __launch_bounds__(spinsim::kEvolveThreadsMax, 2) '
                f"spinsim_evolve_user(spinsim::EvolveArgs a) {{\n"
                f"    spinsim::evolve_body<{tmpl(v, 0)}>(a);\n}}\n")
        write_if_changed(src, body)
        units.append(("lto", name, src))
        reg_decl.append(f'extern "C" const unsigned char spinsim_blob_{name}_begin[], spinsim_blob_{name}_end[];')
        user_rows.append(f"    {{{v[0]}, {v[1]}, {v[2]}, {v[3]}, {v[4]}, spinsim_blob_{name}_begin, "
                         f"spinsim_blob_{name}_end}},")
    # FP32-bulk tone kernels with the field samples on the FP64 tensor path (one per spin mix and
    # register budget; the exponentiators do not enter them).
    dmma_rows = []
    for dims in (0, 2, 3):
        for minb in DMMA_MINB:
            name = f"dmma_d{dims}_b{minb}"
            src = os.path.join(GEN, f"k_{name}.cu")
            body = (f'#include "evolve_dmma.cuh"\n'
                    f"namespace spinsim {{\ntemplate __global__ void evolve_dmma_kernel<{dims}, {minb}>(EvolveArgs);\n}}\n"
                    f'extern "C" const void* spinsim_kget_{name}(void) {{\n'
                    f"    return (const void*)&spinsim::evolve_dmma_kernel<{dims}, {minb}>;\n}}\n")
            write_if_changed(src, body)
            units.append(("sass", name, src))
            reg_decl.append(f'extern "C" const void* spinsim_kget_{name}(void);')
            dmma_rows.append(f"    {{{dims}, {minb}, spinsim_kget_{name}}},")
    # the tensor path's per-instance constants (one small launch before the time evolution)
    src = os.path.join(GEN, "k_dmma_consts.cu")
    write_if_changed(src, '#define SPINSIM_DMMA_CONSTS_KERNEL 1\n#include "evolve_dmma.cuh"\n'
                          'extern "C" const void* spinsim_kget_dmma_consts(void) {\n'
                          '    return (const void*)&spinsim::dmma_consts_kernel;\n}\n')
    units.append(("sass", "dmma_consts", src))
    reg_decl.append('extern "C" const void* spinsim_kget_dmma_consts(void);')
    reg = ("// generated by spinsim_b200/build.py\n" + "\n".join(reg_decl) +
           "\nstatic const BuiltinEntry kBuiltin[] = {\n" + "\n".join(builtin_rows) + "\n};\n"
           "static const UserEntry kUser[] = {\n" + "\n".join(user_rows) + "\n};\n"
           "static const DmmaEntry kDmma[] = {\n" + "\n".join(dmma_rows) + "\n};\n")
    write_if_changed(os.path.join(GEN, "registry_gen.inc"), reg)
    return units


def write_if_changed(path, text):
    if os.path.exists(path) and open(path).read() == text:
        return
    with open(path, "w") as f:
        f.write(text)


def source_digest():
    h = hashlib.sha256()
    for root in (CSRC, INCLUDE):
        for fn in sorted(os.listdir(root)):
            p = os.path.join(root, fn)
            if os.path.isfile(p):
                h.update(fn.encode())
                h.update(open(p, "rb").read())
    return h.hexdigest()


def run_cached(cmd, out, inputs_digest, log):
    stamp = out + ".stamp"
    key = hashlib.sha256((" ".join(cmd) + inputs_digest).encode()).hexdigest()
    if os.path.exists(out) and os.path.exists(stamp) and open(stamp).read() == key:
        return False
    r = subprocess.run(cmd, capture_output=True, text=True)
    with open(log, "w") as f:
        f.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
    if r.returncode != 0:
        raise RuntimeError(f"build step failed ({out}):\n{r.stderr[-4000:]}")
    with open(stamp, "w") as f:
        f.write(key)
    return True


def build(jobs=None, force=False, verbose=False):
    """Compile every CUDA unit for sm_100a and link libspinsim_b200.so.  Returns the library path."""
    os.makedirs(BUILD, exist_ok=True)
    if force:
        for fn in os.listdir(BUILD):
            if fn.endswith(".stamp"):
                os.remove(os.path.join(BUILD, fn))
    units = gen_sources()
    digest = source_digest()
    nv = nvcc()
    tasks = []
    objects, blobs = [], []
    for kind, name, src in units:
        gdig = digest + open(src).read()
        if kind == "sass":
            out = os.path.join(BUILD, f"k_{name}.o")
            cmd = [nv, ARCH_SASS, *COMMON, "-Xptxas", "-v", "-c", src, "-o", out]
            objects.append(out)
        else:
            out = os.path.join(BUILD, f"u_{name}.fatbin")
            cmd = [nv, ARCH_LTO, *COMMON, "-rdc=true", "-fatbin", src, "-o", out]
            blobs.append((name, out))
        tasks.append((cmd, out, gdig, out + ".log"))
    capi_o = os.path.join(BUILD, "capi.o")
    tasks.append(([nv, ARCH_SASS, *COMMON, "-Xptxas", "-v", "-c", os.path.join(CSRC, "capi.cu"), "-o", capi_o],
                  capi_o, digest + open(os.path.join(GEN, "registry_gen.inc")).read(), capi_o + ".log"))
    objects.append(capi_o)
    jobs = jobs or os.cpu_count() or 4
    changed = False
    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        futs = [ex.submit(run_cached, *t) for t in tasks]
        for f in futs:
            changed |= f.result()
    # Embed the LTO fatbins.
    asm = os.path.join(GEN, "blobs.S")
    lines = ['.section .note.GNU-stack,"",@progbits', ".section .rodata"]
    for name, path in blobs:
        lines += [".balign 64", f".global spinsim_blob_{name}_begin", f"spinsim_blob_{name}_begin:",
                  f'.incbin "{path}"', f".global spinsim_blob_{name}_end", f"spinsim_blob_{name}_end:",
                  ".byte 0"]
    write_if_changed(asm, "\n".join(lines) + "\n")
    blobs_o = os.path.join(BUILD, "blobs.o")
    blob_digest = hashlib.sha256(b"".join(open(p, "rb").read() for _, p in blobs)).hexdigest()
    changed |= run_cached([host_cc(), "-c", asm, "-o", blobs_o], blobs_o, blob_digest + open(asm).read(),
                          blobs_o + ".log")
    objects.append(blobs_o)
    if changed or not os.path.exists(LIB):
        tmp = LIB + ".tmp"
        cmd = [nv, ARCH_SASS, "-shared", "-Xcompiler", "-fPIC", "-o", tmp, *objects, "-ldl"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stderr[-4000:]}")
        os.replace(tmp, LIB)
    if verbose:
        print(LIB)
    return LIB


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("-j", type=int, default=None)
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    build(a.j, a.force, verbose=True)


if __name__ == "__main__":
    sys.exit(main())
