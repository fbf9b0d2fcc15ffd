"""Build recipe for the reference interpreter used as the CPU oracle.

Compiles the reference's own C++ sources (the same object lists its per-directory
Makefiles name, e.g. runtime/Makefile, interp/Makefile) where they lie under the
reference checkout, with g++ -O2 as Makefile.common:5-6 does, against the
declaration-only OpenCL header in oracle/clshim and the failing stubs in
oracle/clstub.c.  The OpenCL back end therefore finds no platform and every
trace runs on the reference's CPU interpreter device.

Outputs go only to oracle/_ref/ (git-ignored):
  oracle/_ref/libchai_ref.so   the reference library (interpreter path)
  oracle/_ref/include/chai/    symlinks to the reference's public headers
  oracle/_ref/ref_driver       the trace driver built from oracle/ref_driver.cpp
  oracle/_ref/libr123_jit.so   the Random123 bijections exactly as the reference
                               JIT prints them (oracle/r123_gen.cpp), as C++
  oracle/_ref/libr123_upstream.so  the vendored upstream Random123 OpenCL text
                               (Random123/r123*.i) compiled as C++

Test infrastructure only: the product never links or runs anything built here.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import re
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT = HERE / "_ref"
# The reference checkout: the CHAI_REFERENCE environment variable or
# set_reference() (the command line's --reference).  There is no built-in
# default; without one, only the oracle's own restatement is built.
_ref_env = os.environ.get("CHAI_REFERENCE")
REF = Path(_ref_env) if _ref_env else None


def set_reference(path) -> None:
    global REF
    REF = Path(path) if path else None

# Directory order of the reference's top-level Makefile `all` target
# (Makefile:3-24), minus tools_ (CLI programs) and with vendor built from
# Makefile.NVIDIA's object list.
DIRS = ["misc", "Random123", "vendor", "autotune", "kernel", "bytecode", "common",
        "memmgr", "interp", "jitast", "jitbc", "jitstmt", "jitkrnl", "enqueue",
        "runtime", "api", "applib"]
PUBLIC_HEADERS = {"chai.h": "api", "BC.hpp": "bytecode", "RefCnt.hpp": "bytecode",
                  "Stak.hpp": "bytecode", "Visit.hpp": "bytecode"}


def _objects(d: Path) -> list[str]:
    mk = d / ("Makefile.NVIDIA" if d.name == "vendor" else "Makefile")
    text = mk.read_text()
    m = re.search(r"LIBRARY_OBJECT_CODE\s*=\s*((?:.*\\\n)*.*)", text)
    if not m:
        return []
    names = re.findall(r"([A-Za-z0-9_]+)\.o", m.group(1))
    return [n + ".cpp" for n in names]


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("command failed: %s\n%s" % (" ".join(cmd), r.stderr[-4000:]))


# Files compiled without optimisation and without unreachable traps:
# ArrayBase::assignOther and ArrayBase::assignExp (api/ArrayBase.cpp:122-143)
# return ArrayBase& but end without a return statement.  GCC 13 treats the end
# of such a function as unreachable (a trap instruction at -O0, anything at
# -O1 and above), so every `array = expression` assignment of a sample program
# crashes.  At -O0 with -fno-unreachable-traps the function simply returns;
# its callers (api/ArrayFP.cpp:42,49) ignore the value.
O0_FILES = {("api", "ArrayBase.cpp")}


def available() -> bool:
    return REF is not None and (REF / "api" / "chai.h").exists()


def build(force: bool = False) -> Path:
    """Compile the reference interpreter library and the trace driver."""
    if not available():
        raise FileNotFoundError("reference sources not found at %s" % REF)
    lib = OUT / "libchai_ref.so"
    drv = OUT / "ref_driver"
    drv_src = HERE / "ref_driver.cpp"
    if not force and lib.exists() and drv.exists() and drv.stat().st_mtime >= drv_src.stat().st_mtime and \
            lib.stat().st_mtime >= HERE.joinpath("build_ref.py").stat().st_mtime:
        return OUT
    objdir = OUT / "obj"
    objdir.mkdir(parents=True, exist_ok=True)
    inc = OUT / "include" / "chai"
    inc.mkdir(parents=True, exist_ok=True)
    for name, d in PUBLIC_HEADERS.items():
        link = inc / name
        if link.is_symlink() or link.exists():
            link.unlink()
        link.symlink_to(REF / d / name)
    incs = ["-I" + str(HERE / "clshim"), "-I" + str(OUT / "include")]
    incs += ["-I" + str(REF / d) for d in DIRS]
    flags = ["-O2", "-fPIC", "-fopenmp", "-w", "-std=gnu++98", "-include", "cstddef",
             "-D_VENDOR_IS_NVIDIA_", "-D__STDC_LIMIT_MACROS"]
    jobs = []
    for d in DIRS:
        for src in _objects(REF / d):
            obj = objdir / (d + "__" + src.replace(".cpp", ".o"))
            if force or not obj.exists() or (d, src) in O0_FILES and obj.stat().st_mtime < HERE.joinpath(
                    "build_ref.py").stat().st_mtime:
                fl = [("-O0" if f == "-O2" else f) for f in flags] + ["-fno-unreachable-traps"] \
                    if (d, src) in O0_FILES else flags
                jobs.append(["g++", "-c", *fl, *incs, str(REF / d / src), "-o", str(obj)])
    with cf.ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as ex:
        list(ex.map(_run, jobs))
    stub = objdir / "clstub.o"
    _run(["gcc", "-c", "-O2", "-fPIC", "-I" + str(HERE / "clshim"), str(HERE / "clstub.c"), "-o", str(stub)])
    objs = sorted(str(p) for p in objdir.glob("*.o"))
    _run(["g++", "-shared", "-fopenmp", "-o", str(lib), *objs, "-lpthread"])
    _run(["g++", "-O2", "-fopenmp", "-std=gnu++11", "-I" + str(OUT / "include"), str(drv_src),
          "-o", str(drv), "-L" + str(OUT), "-lchai_ref", "-Wl,-rpath,$ORIGIN", "-lpthread"])
    return OUT


# C++ spellings of the OpenCL built-ins the Random123 text uses.
_R123_PRELUDE = """#include <stdint.h>
typedef uint64_t ulong;
static inline uint64_t mul_hi(uint64_t a, uint64_t b)
{ return (uint64_t)(((unsigned __int128)a * (unsigned __int128)b) >> 64); }
"""

# extern "C" entry points over the generated / upstream generator functions.
_R123_EXPORTS = """
extern "C" {
#define EXP2(NAME, W, KW) void PFX_##NAME(const W* c, const W* k, W* o) { \\
    NAME##_ctr_t C; NAME##_key_t K; for (int i = 0; i < 2; i++) C.v[i] = c[i]; \\
    for (int i = 0; i < KW; i++) K.v[i] = k[i]; NAME##_ctr_t R = NAME##_R(NAME##_rounds, C, K); \\
    for (int i = 0; i < 2; i++) o[i] = R.v[i]; }
#define EXP4(NAME, W, KW) void PFX_##NAME(const W* c, const W* k, W* o) { \\
    NAME##_ctr_t C; NAME##_key_t K; for (int i = 0; i < 4; i++) C.v[i] = c[i]; \\
    for (int i = 0; i < KW; i++) K.v[i] = k[i]; NAME##_ctr_t R = NAME##_R(NAME##_rounds, C, K); \\
    for (int i = 0; i < 4; i++) o[i] = R.v[i]; }
EXP2(philox2x32, uint32_t, 1)
EXP4(philox4x32, uint32_t, 2)
EXP2(philox2x64, uint64_t, 1)
EXP2(threefry2x32, uint32_t, 2)
EXP4(threefry4x32, uint32_t, 4)
EXP2(threefry2x64, uint64_t, 2)
}
"""


def _strip_wrappers(text: str) -> str:
    """Keep the bijections of the JIT's Random123 text: drop the OpenCL
    integer typedefs and the *_uniform_* / *_normal_* wrappers, which use
    OpenCL vector types (R123Philox.cpp:288-523, R123Threefry.cpp:289-535)."""
    out, skipping = [], False
    wrapper = re.compile(r"^inline \S+ (philox|threefry)_(uniform|normal)_\d+_\d+\(")
    for line in text.splitlines():
        if skipping:
            if line.strip() == "}":
                skipping = False
            continue
        if line.startswith("typedef ulong") or line.startswith("typedef uint ") or \
                line.startswith("typedef uchar"):
            continue
        if wrapper.match(line):
            if line.rstrip().endswith("{"):
                skipping = True
            continue
        out.append(line)
    return "\n".join(out) + "\n"


def build_r123_pins(force: bool = False) -> None:
    """Compile the reference JIT's generated Random123 text and the vendored
    upstream Random123 OpenCL text as C++ libraries (oracle/_ref)."""
    jit_so, up_so = OUT / "libr123_jit.so", OUT / "libr123_upstream.so"
    if not force and jit_so.exists() and up_so.exists():
        return
    gen = OUT / "r123_gen"
    _run(["g++", "-O1", "-std=gnu++98", "-include", "cstddef", "-I" + str(REF / "Random123"),
          "-I" + str(REF / "misc"), str(HERE / "r123_gen.cpp"), "-o", str(gen), "-L" + str(OUT),
          "-lchai_ref", "-Wl,-rpath,$ORIGIN", "-fopenmp"])
    text = subprocess.run([str(gen)], capture_output=True, text=True, check=True).stdout
    (OUT / "r123_jit.cl").write_text(text)
    src = _R123_PRELUDE + _strip_wrappers(text) + _R123_EXPORTS.replace("PFX_", "jit_")
    (OUT / "r123_jit.cpp").write_text(src)
    _run(["g++", "-O2", "-fPIC", "-shared", "-w", str(OUT / "r123_jit.cpp"), "-o", str(jit_so)])
    up = OUT / "r123_upstream.cpp"
    up.write_text(_R123_PRELUDE + "\n".join(
        '#include "%s"' % (REF / "Random123" / n) for n in ("r123array.i", "r123philox.i", "r123threefry.i"))
        + "\n" + _R123_EXPORTS.replace("PFX_", "up_"))
    _run(["g++", "-O2", "-fPIC", "-shared", "-w", str(up), "-o", str(up_so)])


# C spellings (GCC vector extensions) of the OpenCL vector types and built-ins
# the generated wrappers use.
_VEC_TYPES = {"uint": ("uint32_t", (2, 4)), "int": ("int32_t", (2, 4)), "float": ("float", (2, 4)),
              "ulong": ("uint64_t", (2, 4)), "long": ("int64_t", (2, 4)), "double": ("double", (2, 4))}


def _wrap_prelude() -> str:
    lines = ["#include <stdint.h>", "#include <string.h>", "#include <tgmath.h>",
             "typedef uint32_t uint; typedef uint64_t ulong; typedef unsigned char uchar;",
             "static inline uint64_t mul_hi(uint64_t a, uint64_t b)",
             "{ return (uint64_t)(((unsigned __int128)a * (unsigned __int128)b) >> 64); }"]
    for name, (ct, widths) in _VEC_TYPES.items():
        for n in widths:
            t = "%s%d" % (name, n)
            lines.append("typedef %s %s __attribute__((vector_size(%d * sizeof(%s))));" % (ct, t, n, ct))
            lines.append("#define VEC_%s_1(x) ((%s){%s})" % (t, t, ", ".join(["(x)"] * n)))
            args = ", ".join("a%d" % i for i in range(n))
            lines.append("#define VEC_%s_%d(%s) ((%s){%s})" % (t, n, args, t, ", ".join("(a%d)" % i for i in range(n))))
    return "\n".join(lines) + "\n"


def _split_args(text: str, start: int):
    """Top-level argument count of the parenthesised list opening at start."""
    depth, count, i = 0, 1, start
    while True:
        c = text[i]
        if c == "(":
            depth += 1
        elif c == ")":
            depth -= 1
            if depth == 0:
                return count, i
        elif c == "," and depth == 1:
            count += 1
        i += 1


def _opencl_to_c(text: str) -> str:
    """Rewrite the generated OpenCL generator text as C: vector casts and
    literals, .sN components, convert_* built-ins, static inline functions."""
    text = "\n".join(l for l in text.splitlines()
                     if not re.match(r"typedef (ulong|uint|uchar) uint(64|32|8)_t;", l))
    text = re.sub(r"^inline ", "static inline ", text, flags=re.M)
    text = re.sub(r"\.s([0-3])\b", r"[\1]", text)
    text = re.sub(r"convert_(float|double)\(", r"(\1)(", text)
    text = re.sub(r"convert_((?:float|double)[24])\(([^()]*(?:\([^()]*\))?[^()]*)\)",
                  r"__builtin_convertvector((\2), \1)", text)
    pat = re.compile(r"\(((?:u?int|float|u?long|double)[24])\)\(")
    out, pos = [], 0
    for m in pat.finditer(text):
        if m.start() < pos:
            continue
        n, _ = _split_args(text, m.end() - 1)
        out.append(text[pos:m.start()])
        out.append("VEC_%s_%d(" % (m.group(1), n))
        pos = m.end()
    out.append(text[pos:])
    return "".join(out)


def build_r123_wrapper_pins(force: bool = False) -> Path:
    """Compile the reference JIT's complete generated Random123 text -- the
    bijections and chai's per-variant uniform / normal wrappers with their
    key / counter layout (Random123/R123Philox.cpp:288-523,
    Random123/R123Threefry.cpp:289-535) -- as C with GCC vector types, and
    export every wrapper as w_<name>(tid, idx, out)."""
    so = OUT / "libr123_wrappers.so"
    src_cl = OUT / "r123_jit.cl"
    if not force and so.exists() and so.stat().st_mtime >= src_cl.stat().st_mtime:
        return so
    text = src_cl.read_text()
    exports = []
    for m in re.finditer(r"^inline (\w+) ((?:philox|threefry)_(?:uniform|normal)_\d+_\d+)\((uint(?:32|64)_t) tid, "
                         r"\w+ idx\) \{", text, flags=re.M):
        rt, name, at = m.groups()
        exports.append("void w_%s(uint64_t tid, uint64_t idx, void* out) { %s r = %s((%s)tid, (%s)idx); "
                       "memcpy(out, &r, sizeof r); }" % (name, rt, name, at, at))
    c_src = OUT / "r123_wrappers.c"
    c_src.write_text(_wrap_prelude() + _opencl_to_c(text) + "\n" + "\n".join(exports) + "\n")
    _run(["gcc", "-O1", "-fPIC", "-shared", "-w", "-std=gnu11", "-ffp-contract=off", str(c_src), "-o", str(so),
          "-lm"])
    return so


# Reference sample programs run unchanged on the B200 through the reference's
# own front end and chai_b200's CudaDevice (source file -> macros it needs).
SAMPLES = {
    "matmul_uni": "sample/matmul_uni.cpp", "matmul_vec": "sample/matmul_vec.cpp",
    "matmul_pth": "sample/matmul_pth.cpp", "matmul64_uni": "sample/matmul64_uni.cpp",
    "sum_uni": "sample/sum_uni.cpp", "sum_vec": "sample/sum_vec.cpp", "sum_pth": "sample/sum_pth.cpp",
    "loopsum_uni": "sample/loopsum_uni.cpp", "loopsum_vec": "sample/loopsum_vec.cpp",
    "cg": "sample/cg.cpp", "cg64": "sample/cg64.cpp", "index": "sample/index.cpp", "md5": "sample/md5.cpp",
    "mingle": "sample/mingle.cpp", "filter": "sample/filter.cpp", "kirch": "sample/kirch.cpp",
    "pi": "sample/pi.cpp", "inline_cl": "sample/inline_cl.cpp",
    "american_option": "sample/finance/american_option.cpp",
    "american_option_batch": "sample/finance/american_option_batch.cpp",
    "bitonic": "sample/sorting/bitonic.cpp",
}
CUDA_OUT = OUT / "cuda"
LIBCHAI_B200 = HERE.parent / "chai_b200" / "libchai_b200.so"


def build_cuda_frontend(force: bool = False) -> Path:
    """The reference's front end linked with chai_b200 through the CudaDevice
    adapter (chai_b200/refdevice/): every reference object except
    runtime/DeviceMap.cpp, whose place the adapter's DeviceMap.cpp takes, into
    oracle/_ref/cuda/libchai_ref_cuda.so; then the reference's sample programs,
    unchanged, linked against it (oracle/_ref/cuda/<sample>).  A sample runs on
    the reference interpreter as usual, and on the B200 when CHAI_CUDA is set.
    Needs the reference objects from build() and libchai_b200.so."""
    build()
    CUDA_OUT.mkdir(parents=True, exist_ok=True)
    objdir = OUT / "obj"
    inc = CUDA_OUT / "include" / "chai"
    inc.mkdir(parents=True, exist_ok=True)
    for name, d in dict(PUBLIC_HEADERS, **{"ParseArgs.hpp": "applib"}).items():
        link = inc / name
        if link.is_symlink() or link.exists():
            link.unlink()
        link.symlink_to(REF / d / name)
    adapter = HERE.parent / "chai_b200" / "refdevice"
    incs = ["-I" + str(adapter), "-I" + str(HERE.parent / "include"), "-I" + str(HERE / "clshim"),
            "-I" + str(OUT / "include")] + ["-I" + str(REF / d) for d in DIRS]
    flags = ["-O2", "-fPIC", "-fopenmp", "-w", "-std=gnu++98", "-include", "cstddef",
             "-D_VENDOR_IS_NVIDIA_", "-D__STDC_LIMIT_MACROS"]
    lib = CUDA_OUT / "libchai_ref_cuda.so"
    srcs = [adapter / "CudaDevice.cpp", adapter / "DeviceMap.cpp"]
    newest = max([x.stat().st_mtime for x in srcs + [adapter / "CudaDevice.hpp", HERE.parent / "include" /
                                                      "chai_b200.h"]])
    if force or not lib.exists() or lib.stat().st_mtime < newest:
        objs = []
        for src in srcs:
            o = CUDA_OUT / (src.stem + ".o")
            _run(["g++", "-c", *flags, *incs, str(src), "-o", str(o)])
            objs.append(str(o))
        ref_objs = sorted(str(x) for x in objdir.glob("*.o") if x.name != "runtime__DeviceMap.o")
        rpath = "-Wl,-rpath,$ORIGIN/../../../chai_b200"
        _run(["g++", "-shared", "-fopenmp", "-o", str(lib), *ref_objs, *objs, "-L" + str(LIBCHAI_B200.parent),
              "-lchai_b200", rpath, "-lpthread"])
    for name, rel in SAMPLES.items():
        exe = CUDA_OUT / name
        src = REF / rel
        if not force and exe.exists() and exe.stat().st_mtime >= lib.stat().st_mtime:
            continue
        _run(["g++", "-O2", "-fopenmp", "-w", "-std=gnu++98", "-include", "cstddef", "-I" + str(CUDA_OUT / "include"),
              "-I" + str(src.parent), str(src), "-o", str(exe), "-L" + str(CUDA_OUT), "-lchai_ref_cuda",
              "-L" + str(LIBCHAI_B200.parent), "-lchai_b200", "-Wl,-rpath,$ORIGIN",
              "-Wl,-rpath,$ORIGIN/../../../chai_b200", "-lpthread"])
    return CUDA_OUT


def build_all() -> None:
    """Everything the oracle pins need that this host can build."""
    build_oracle()
    if available():
        build()
        build_r123_pins()
        build_r123_wrapper_pins()
        if LIBCHAI_B200.exists():
            build_cuda_frontend()


def build_oracle() -> Path:
    """Compile the oracle's own C restatement (always possible; no reference
    sources needed) into oracle/_build/liboracle.so."""
    bdir = HERE / "_build"
    bdir.mkdir(exist_ok=True)
    so = bdir / "liboracle.so"
    srcs = [HERE / "r123.c", HERE / "ops.c"]
    if not so.exists() or any(s.stat().st_mtime > so.stat().st_mtime for s in srcs):
        _run(["gcc", "-O2", "-fPIC", "-shared", "-fopenmp", "-std=gnu11", *map(str, srcs),
              "-o", str(so), "-lm"])
    return so


if __name__ == "__main__":
    if "--reference" in sys.argv:
        set_reference(sys.argv[sys.argv.index("--reference") + 1])
    build_oracle()
    build(force="--force" in sys.argv)
    build_r123_pins(force="--force" in sys.argv)
    build_r123_wrapper_pins(force="--force" in sys.argv)
    print(OUT)
