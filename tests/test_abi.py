"""The C ABI boundary, checked without a GPU: the library loads, exports every
function include/mfista_b200.h declares, and struct RESULT is laid out as in
the reference header (c/mfista.h:45-66).  No compute call is made here."""
import ctypes as C
import os
import re
import subprocess

import pytest

from conftest import REFERENCE_C, ROOT

HEADER = os.path.join(ROOT, "include", "mfista_b200.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"\b(mfista_\w+)\s*\(", text)
    return sorted(set(names))


def test_library_exports_every_declared_symbol():
    from sparseimaging_b200 import build
    build.build(verbose=False)
    lib = C.CDLL(build.LIB)
    names = declared_functions()
    assert "mfista_imaging_core_nufft" in names and len(names) >= 18
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_exported_symbols_are_declared():
    from sparseimaging_b200 import build
    out = subprocess.run(["nm", "-D", "--defined-only", build.LIB], capture_output=True, text=True).stdout
    exported = sorted(set(re.findall(r" T (mfista_\w+)", out)))
    assert set(exported) <= set(declared_functions())


PROBE = r"""
#include <stdio.h>
#include <stddef.h>
#include "HDR"
int main(void) {
  printf("%zu", sizeof(struct RESULT));
#define F(x) printf(" %zu", offsetof(struct RESULT, x));
  F(M) F(N) F(NX) F(NY) F(N_active) F(maxiter) F(ITER) F(nonneg) F(lambda_l1) F(lambda_tv)
  F(lambda_tsv) F(sq_error) F(mean_sq_error) F(l1cost) F(tvcost) F(tsvcost) F(finalcost)
  F(comp_time) F(residual) F(Lip_const)
  printf("\n");
  return 0;
}
"""


def _layout(header, tmp_path, extra_inc=()):
    src = tmp_path / "probe.c"
    src.write_text(PROBE.replace("HDR", header))
    exe = tmp_path / "probe"
    cmd = ["gcc", "-o", str(exe), str(src)] + [f"-I{d}" for d in extra_inc]
    subprocess.run(cmd, check=True, capture_output=True)
    return [int(v) for v in subprocess.run([str(exe)], capture_output=True, text=True).stdout.split()]


def test_result_layout_matches_ctypes(tmp_path):
    from sparseimaging_b200 import RESULT
    got = _layout(HEADER, tmp_path)
    want = [C.sizeof(RESULT)] + [getattr(RESULT, f).offset for f, _ in RESULT._fields_]
    assert got == want


@pytest.mark.skipif(not os.path.isdir(REFERENCE_C), reason="reference sources not present")
def test_result_layout_matches_reference_header(tmp_path):
    ours = _layout(HEADER, tmp_path)
    ref = _layout(os.path.join(REFERENCE_C, "mfista.h"), tmp_path,
                  extra_inc=[os.path.join(ROOT, "oracle", "shim"), REFERENCE_C])
    assert ours == ref


def test_entry_point_signatures_match_reference(tmp_path):
    """Compiles a translation unit that declares the reference prototypes
    (c/mfista.h:151-178, restated) next to ours: conflicting types fail."""
    src = tmp_path / "sig.c"
    src.write_text('#include "%s"\n' % HEADER + r"""
void mfista_imaging_core_dft(double *y, double *A, int *M, int *N, int NX, int NY, int maxiter,
  double eps, double lambda_l1, double lambda_tv, double lambda_tsv, double cinit, double *xinit,
  double *xout, int nonneg_flag, int looe_flag, int box_flag, float *cl_box, struct RESULT *r);
void mfista_imaging_core_fft(int *u_idx, int *v_idx, double *y_r, double *y_i, double *noise_stdev,
  int M, int NX, int NY, int maxiter, double eps, double lambda_l1, double lambda_tv,
  double lambda_tsv, double cinit, double *xinit, double *xout, int nonneg_flag,
  unsigned int fftw_plan_flag, int box_flag, float *cl_box, struct RESULT *r);
void mfista_imaging_core_nufft(double *u_dx, double *v_dy, double *vis_r, double *vis_i,
  double *vis_std, int M, int NX, int NY, int maxiter, double eps, double lambda_l1,
  double lambda_tv, double lambda_tsv, double cinit, double *xinit, double *xout,
  int nonneg_flag, int box_flag, float *cl_box, struct RESULT *r);
int main(void) { return 0; }
""")
    subprocess.run(["gcc", "-Werror", "-o", str(tmp_path / "sig"), str(src)], check=True)


def test_python_binding_raises_without_library(monkeypatch, tmp_path):
    import sparseimaging_b200 as si
    monkeypatch.setattr(si, "LIB", str(tmp_path / "missing.so"))
    monkeypatch.setattr(si, "_lib", None)
    with pytest.raises(RuntimeError):
        si.lib()


def test_cpp_build_shim_links(tmp_path):
    """A one-line shim that gives programs written against the reference's
    C++ build its x2y_nufft (c++/mfista.hpp:136-137) compiles against our
    header and links against the library (nothing is run)."""
    from sparseimaging_b200 import build
    src = tmp_path / "shim.c"
    src.write_text('#include "%s"\n' % HEADER + r"""
void x2y_nufft(double *u_dx, double *v_dy, int M, int Nx, int Ny,
               double *xin, double *y_r, double *y_i)
{ mfista_cpp_x2y_nufft(u_dx, v_dy, M, Nx, Ny, xin, y_r, y_i); }
int main(int argc, char **argv) { if (argc > 99) x2y_nufft(0, 0, 0, 0, 0, 0, 0, 0); return 0; }
""")
    libdir = os.path.dirname(build.LIB)
    subprocess.run(["gcc", "-Werror", "-o", str(tmp_path / "shim"), str(src), f"-L{libdir}",
                    f"-l:{os.path.basename(build.LIB)}", f"-Wl,-rpath,{libdir}"], check=True)


def test_cpp_build_library_exports_the_cpp_names():
    """libmfista_b200_cpp.so exports the names of the reference's C++ build
    (c++/mfista.hpp:115-140) declared in include/mfista_b200_cpp.h."""
    from sparseimaging_b200 import build
    build.build(verbose=False)
    hdr = open(os.path.join(ROOT, "include", "mfista_b200_cpp.h")).read()
    hdr = re.sub(r"/\*.*?\*/", "", hdr, flags=re.S)
    names = sorted(set(re.findall(r"\b(\w+)\s*\(", hdr)))
    assert names == ["mfista_imaging_core_fft", "mfista_imaging_core_nufft", "x2y_nufft", "y2x_nufft"]
    out = subprocess.run(["nm", "-D", "--defined-only", build.CPP_LIB], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (\w+)", out))
    assert set(names) <= exported
    lib = C.CDLL(build.CPP_LIB)
    for n in names:
        assert hasattr(lib, n)
