"""Build helper for the C++ drop-in caller (caller.cpp)."""
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")


def build_caller(outdir: str) -> str:
    """Compile caller.cpp against include/nspb_compat.h, linking libnspb.so,
    cudart and cuSPARSE (for the descriptor calls CSRm::init/free make)."""
    exe = os.path.join(outdir, "caller")
    lib_dir = os.path.join(ROOT, "nsp_b200")
    cmd = ["g++", "-std=c++17", "-O1", "-Wall", "-Wextra", "-o", exe,
           os.path.join(HERE, "caller.cpp"), "-I", os.path.join(ROOT, "include"),
           "-I", os.path.join(CUDA, "include"), "-L", lib_dir, "-lnspb",
           "-L", os.path.join(CUDA, "lib64"), "-lcusparse", "-lcudart",
           f"-Wl,-rpath,{lib_dir}", f"-Wl,-rpath,{os.path.join(CUDA, 'lib64')}"]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return exe
