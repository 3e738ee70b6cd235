"""The C++ drop-in caller (tests/dropin/caller.cpp) compiles and links
against include/nspb_compat.h and libnspb.so with the reference's own
signatures: CSR, nsparseMGPU_version1 and nsp_spgemm_kernel_hash."""
import os

from dropin import build_caller


def test_dropin_caller_builds(tmp_path):
    exe = build_caller(str(tmp_path))
    assert os.access(exe, os.X_OK)


def test_null_descriptor_passes_csrm_free(tmp_path):
    """The CSR the shims return carries a NULL cuSPARSE descriptor; the
    reference's CSRm::free (src/CSR.cu:592) runs
    CHECK_CUSPARSE(cusparseDestroyMatDescr(*A->descr)) on it. That call is
    host-only: run it here and require CUSPARSE_STATUS_SUCCESS."""
    import subprocess
    from dropin import CUDA
    src = tmp_path / "d.cpp"
    src.write_text("#include <cusparse.h>\nint main(){cusparseMatDescr_t d = nullptr;"
                   "return (int)cusparseDestroyMatDescr(d);}\n")
    exe = str(tmp_path / "d")
    subprocess.run(["g++", str(src), "-I", f"{CUDA}/include", "-L", f"{CUDA}/lib64",
                    "-lcusparse", f"-Wl,-rpath,{CUDA}/lib64", "-o", exe], check=True)
    assert subprocess.run([exe]).returncode == 0
