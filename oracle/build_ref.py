"""Build the reference CUDA rasterizer extension from its own sources into oracle/_ref/.

Test and benchmark infrastructure only. Compiles the reference's cuda/binding.cpp,
cuda/forward.cu, cuda/backward.cu and cuda/raster.cu (as the reference's
cuda/rasterizer.py:20-33 does, but for sm_100a) with torch.utils.cpp_extension,
reading the sources where they lie in the reference checkout and writing only
under oracle/_ref/. The resulting qpf_2d_cuda*.so is the GPU reference arm of
the benchmark and a second checker for the tile lists; it is never used by
the product package. Needs nvcc; no GPU.

    python oracle/build_ref.py [--reference DIR]

The reference checkout is taken from --reference, else from the environment
variable CVQPG_REFERENCE_DIR, else from the read-only checkout location of the
build machine (this recipe is the one place that names it). Without sources it
prints why and exits 0, so build() works where the reference is absent.
"""
import glob
import os
import shutil
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
BUILD_MACHINE_CHECKOUT = "/root/reference"


def reference_dir(argv=None):
    argv = sys.argv[1:] if argv is None else argv
    if "--reference" in argv:
        return argv[argv.index("--reference") + 1]
    return os.environ.get("CVQPG_REFERENCE_DIR", BUILD_MACHINE_CHECKOUT)


def built_path():
    c = sorted(glob.glob(os.path.join(OUT, "qpf_2d_cuda*.so")))
    return c[0] if c else None


def main(argv=None):
    if built_path():
        print("already built:", built_path())
        return 0
    src_dir = os.path.join(reference_dir(argv), "cuda")
    if not os.path.isdir(src_dir):
        print("reference sources not found (set CVQPG_REFERENCE_DIR or --reference):", src_dir)
        return 0
    os.makedirs(OUT, exist_ok=True)
    os.environ.setdefault("TORCH_CUDA_ARCH_LIST", "10.0a")
    from torch.utils.cpp_extension import load
    build_dir = os.path.join(OUT, "build")
    os.makedirs(build_dir, exist_ok=True)
    load(name="qpf_2d_cuda", sources=[os.path.join(src_dir, f) for f in
                                      ("binding.cpp", "forward.cu", "backward.cu", "raster.cu")],
         extra_cflags=["-O3"], extra_cuda_cflags=["-O3", "--threads=8", "-diag-suppress=20012",
                                                  "--expt-relaxed-constexpr"],
         build_directory=build_dir, verbose=False)
    for so in glob.glob(os.path.join(build_dir, "qpf_2d_cuda*.so")):
        shutil.copy2(so, OUT)
    shutil.rmtree(build_dir, ignore_errors=True)
    print("built:", built_path())
    return 0


if __name__ == "__main__":
    sys.exit(main())
