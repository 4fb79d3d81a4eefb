"""Build recipe for the reference's own CUDA kernels -- TEST INFRASTRUCTURE.

Compiles CuRast's `src/kernels/triangles_visbuffer.cu` and
`src/kernels/resolve.cu` straight from the read-only reference checkout
with NVRTC, for sm_100a, into `oracle/_ref/`:

  ref_tv_native.cubin / ref_resolve_native.cubin
      The reference's own JIT recipe (src/CudaModularProgram.h:133-157:
      --use_fast_math, --extra-device-vectorization, -rdc, -default-device,
      --dlink-time-opt, C++20; nvJitLink -lto -O3 at :365-374).  Used to
      time the reference implementation on the same GPU.

  ref_tv_fastnofma.cubin / ref_resolve_fastnofma.cubin
      The reference's recipe with --fmad=false added after --use_fast_math
      (approximate divisions and square roots, no contracted products), as a
      cubin without link-time optimisation.

  ref_tv_ieee.cubin / ref_resolve_ieee.cubin
      Same sources with IEEE float semantics: --fmad=false (no contraction),
      --prec-div=true, --prec-sqrt=true, --ftz=false, and every
      `__fdividef(a, b)` call in triangles_visbuffer.cu (tv.cu:206-211,249)
      rewritten in memory to an IEEE division.  Under these flags the
      reference's visbuffer is a pure function of its inputs, which is what
      the bit-exact parity tests compare against.

The source text is read at build time only; nothing from the reference is
copied into this repository.  Outputs go to oracle/_ref/ (git-ignored, but
shipped with the working tree so the GPU tests can load them).

Usage:  python oracle/build_ref.py [--reference DIR] [--force]
        (DIR defaults to $CURAST_REFERENCE, else /root/reference)
"""
import argparse
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
ARCH = "sm_100a"
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")

IEEE_PRELUDE = (
    "__device__ __forceinline__ float __oracle_ieee_div(float a, float b) { return a / b; }\n"
)


def _lib(name):
    import ctypes
    return ctypes.CDLL(os.path.join(CUDA_HOME, "lib64", name))


def _nvrtc_compile(src: str, name: str, opts, want_ltoir: bool):
    """NVRTC from the CUDA toolkit (not a pip wheel), via ctypes."""
    import ctypes

    lib = _lib("libnvrtc.so")
    prog = ctypes.c_void_p()
    rc = lib.nvrtcCreateProgram(ctypes.byref(prog), src.encode(), name.encode(), 0, None, None)
    if rc != 0:
        raise RuntimeError(f"nvrtcCreateProgram failed: {rc}")
    copts = (ctypes.c_char_p * len(opts))(*[o.encode() for o in opts])
    rc = lib.nvrtcCompileProgram(prog, len(opts), copts)
    n = ctypes.c_size_t()
    lib.nvrtcGetProgramLogSize(prog, ctypes.byref(n))
    log = ctypes.create_string_buffer(n.value)
    lib.nvrtcGetProgramLog(prog, log)
    if rc != 0:
        raise RuntimeError(f"NVRTC failed for {name} ({rc}):\n{log.value.decode(errors='replace')}")
    sz = ctypes.c_size_t()
    if want_ltoir:
        lib.nvrtcGetLTOIRSize(prog, ctypes.byref(sz))
        buf = ctypes.create_string_buffer(sz.value)
        lib.nvrtcGetLTOIR(prog, buf)
    else:
        lib.nvrtcGetCUBINSize(prog, ctypes.byref(sz))
        buf = ctypes.create_string_buffer(sz.value)
        lib.nvrtcGetCUBIN(prog, buf)
    lib.nvrtcDestroyProgram(ctypes.byref(prog))
    return buf.raw[: sz.value]


def _jitlink(ltoir: bytes, name: str) -> bytes:
    """nvJitLink from the CUDA toolkit: LTO link with libcudadevrt."""
    import ctypes

    lib = _lib("libnvJitLink.so")
    opts = ["-lto", f"-arch={ARCH}", "-O3", "-optimize-unused-variables", "-split-compile=0"]
    copts = (ctypes.c_char_p * len(opts))(*[o.encode() for o in opts])
    h = ctypes.c_void_p()
    # nvJitLinkCreate is versioned in the 12.x headers
    create = getattr(lib, "__nvJitLinkCreate_12_9", None) or lib.nvJitLinkCreate
    rc = create(ctypes.byref(h), len(opts), copts)
    if rc != 0:
        raise RuntimeError(f"nvJitLinkCreate failed: {rc}")

    def chk(rc, what):
        if rc != 0:
            n = ctypes.c_size_t()
            lib.nvJitLinkGetErrorLogSize(h, ctypes.byref(n))
            log = ctypes.create_string_buffer(n.value + 1)
            lib.nvJitLinkGetErrorLog(h, log)
            raise RuntimeError(f"{what} failed ({rc}): {log.value.decode(errors='replace')}")

    try:
        NVJITLINK_INPUT_LTOIR, NVJITLINK_INPUT_ANY = 3, 10
        chk(lib.nvJitLinkAddData(h, NVJITLINK_INPUT_LTOIR, ltoir, len(ltoir), name.encode()), "add ltoir")
        chk(lib.nvJitLinkAddFile(h, NVJITLINK_INPUT_ANY,
                                 os.path.join(CUDA_HOME, "lib64", "libcudadevrt.a").encode()), "add cudadevrt")
        chk(lib.nvJitLinkComplete(h), "complete")
        sz = ctypes.c_size_t()
        chk(lib.nvJitLinkGetLinkedCubinSize(h, ctypes.byref(sz)), "cubin size")
        buf = ctypes.create_string_buffer(sz.value)
        chk(lib.nvJitLinkGetLinkedCubin(h, buf), "cubin")
        return buf.raw[: sz.value]
    finally:
        lib.nvJitLinkDestroy(ctypes.byref(h))


def _includes(ref):
    return [
        f"-I{ref}/src/kernels",
        f"-I{CUDA_HOME}/include",
        # the reference adds <cuda>/include/cccl/cuda/std; CUDA 12.9 keeps it here
        f"-I{CUDA_HOME}/include/cuda/std",
        f"-I{ref}",
        f"-I{ref}/libs",
        f"-I{ref}/src",
    ]


def build(ref: str, force: bool = False) -> None:
    os.makedirs(OUT, exist_ok=True)
    modules = {
        "tv": os.path.join(ref, "src", "kernels", "triangles_visbuffer.cu"),
        "resolve": os.path.join(ref, "src", "kernels", "resolve.cu"),
    }
    common = [
        "--extra-device-vectorization",
        "-lineinfo",
        "-default-device",
        "--std=c++20",
        "--disable-warnings",
    ] + _includes(ref)
    cwd = os.getcwd()
    os.chdir(ref)  # the reference compiles with "-I ./" relative to its root
    try:
        for key, path in modules.items():
            src = open(path).read()
            # native: the reference's own recipe, LTO through nvJitLink
            out = os.path.join(OUT, f"ref_{key}_native.cubin")
            if force or not os.path.exists(out):
                opts = [f"--gpu-architecture=compute_{ARCH[3:]}", "--use_fast_math",
                        "--relocatable-device-code=true", "--dlink-time-opt", "--split-compile=0"] + common
                ltoir = _nvrtc_compile(src, os.path.basename(path), opts, want_ltoir=True)
                cubin = _jitlink(ltoir, os.path.basename(path))
                with open(out, "wb") as fh:
                    fh.write(cubin)
            # fastnofma: the reference's own recipe with --fmad=false added (its
            # fast-math approximations without contracted products), built
            # without link-time optimisation so nothing re-contracts at link
            out = os.path.join(OUT, f"ref_{key}_fastnofma.cubin")
            if force or not os.path.exists(out):
                opts = [f"--gpu-architecture={ARCH}", "--use_fast_math", "--fmad=false"] + common
                cubin = _nvrtc_compile(src, os.path.basename(path), opts, want_ltoir=False)
                with open(out, "wb") as fh:
                    fh.write(cubin)
            # ieee: no contraction, IEEE div/sqrt, __fdividef -> IEEE division
            out = os.path.join(OUT, f"ref_{key}_ieee.cubin")
            if force or not os.path.exists(out):
                src_ieee = IEEE_PRELUDE + src.replace("__fdividef(", "__oracle_ieee_div(")
                opts = [f"--gpu-architecture={ARCH}", "--fmad=false", "--prec-div=true",
                        "--prec-sqrt=true", "--ftz=false"] + common
                cubin = _nvrtc_compile(src_ieee, os.path.basename(path), opts, want_ltoir=False)
                with open(out, "wb") as fh:
                    fh.write(cubin)
    finally:
        os.chdir(cwd)


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("CURAST_REFERENCE", "/root/reference"))
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args(argv)
    if not os.path.isdir(a.reference):
        print("reference checkout not present; keeping prebuilt oracle/_ref", file=sys.stderr)
        return 0
    build(a.reference, a.force)
    print("built:", sorted(os.listdir(OUT)))
    return 0


if __name__ == "__main__":
    sys.exit(main())
