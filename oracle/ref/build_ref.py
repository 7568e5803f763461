"""Build recipe for ``oracle/_ref``: the reference's OWN device kernels, compiled
as host C++ under the work-item emulation shim ``oracle/ref/kernel_emu.hpp``.

TEST INFRASTRUCTURE ONLY (oracle).  Nothing in the shipped engine imports this.

The reference generates its kernel source at run time: ``PaSWAS.Code.get_code``
(pyPaSWAS/Core/PaSWAS.py:85-91) substitutes the batch shape (N_SEQUENCES,
N_TARGETS, X, Y), the scoring matrix and the thresholds into the templates
pyPaSWAS/Core/cuda/default_{variable,direction,score,main}.cu (CUDA backend,
canonical semantics) or pyPaSWAS/Core/ocl/default_*_cpu.cl (OpenCL CPU backend,
the reference's own CPU path).  This recipe calls that very template code from
the read-only reference tree, appends small launcher functions of our own, and
compiles the result with g++ into ``oracle/_ref/<tag>.so``.  Sources are never
copied into this repository; only build outputs land in ``oracle/_ref/``.

Each .so exports ``emu_<kernel>(gx, gy, ...)`` launchers that run a whole grid
of the named reference kernel (see kernel_emu.hpp for the execution model).
"""
import hashlib
import logging
import os
import subprocess
import sys
import warnings

REFERENCE_ROOT = os.environ.get("PASWAS_REFERENCE_ROOT", "/root/reference")
HERE = os.path.dirname(os.path.abspath(__file__))
OUT_DIR = os.path.join(os.path.dirname(HERE), "_ref")

# Direction codes of the reference (pyPaSWAS/Core/__init__.py:7-13).
NO_DIRECTION, UPPER_LEFT, UPPER, LEFT, STOP = 32, 1, 2, 3, 64

_CUDA_LAUNCHERS = r"""
// ---- launchers (ours): one call runs one whole grid of a reference kernel ----
extern "C" void emu_calculateScore(unsigned gx, unsigned gy, void* m, unsigned x, unsigned y,
        unsigned nb, char* s, char* t, void* gmax, void* gdir) {
    emu::launch(gx, gy, SHARED_X, SHARED_Y, [&]() {
        calculateScore((GlobalMatrix*)m, x, y, nb, s, t, (GlobalMaxima*)gmax, (GlobalDirection*)gdir); });
}
extern "C" void emu_calculateScoreAffineGap(unsigned gx, unsigned gy, void* m, void* mi, void* mj,
        unsigned x, unsigned y, unsigned nb, char* s, char* t, void* gmax, void* gdir) {
    emu::launch(gx, gy, SHARED_X, SHARED_Y, [&]() {
        calculateScoreAffineGap((GlobalMatrix*)m, (GlobalMatrix*)mi, (GlobalMatrix*)mj, x, y, nb, s, t,
                                (GlobalMaxima*)gmax, (GlobalDirection*)gdir); });
}
extern "C" void emu_traceback(unsigned gx, unsigned gy, void* m, unsigned x, unsigned y, unsigned nb,
        void* gmax, void* gdir, void* gdirzc, unsigned* idx, void* sp, float* mps) {
    emu::launch(gx, gy, SHARED_X, SHARED_Y, [&]() {
        traceback((GlobalMatrix*)m, x, y, nb, (GlobalMaxima*)gmax, (GlobalDirection*)gdir,
                  (GlobalDirection*)gdirzc, idx, (StartingPoints*)sp, mps); });
}
extern "C" void emu_tracebackAffineGap(unsigned gx, unsigned gy, void* m, void* mi, void* mj,
        unsigned x, unsigned y, unsigned nb, void* gmax, void* gdir, void* gdirzc, unsigned* idx,
        void* sp, float* mps) {
    emu::launch(gx, gy, SHARED_X, SHARED_Y, [&]() {
        tracebackAffineGap((GlobalMatrix*)m, (GlobalMatrix*)mi, (GlobalMatrix*)mj, x, y, nb,
                           (GlobalMaxima*)gmax, (GlobalDirection*)gdir, (GlobalDirection*)gdirzc, idx,
                           (StartingPoints*)sp, mps); });
}
"""

_OCL_CPU_LAUNCHERS = r"""
// ---- launchers (ours) for the OpenCL CPU kernels; nthreads spreads work-groups ----
extern "C" void emu_calculateScore(unsigned gx, unsigned gy, void* m, unsigned x, unsigned y,
        unsigned nb, char* s, char* t, void* gmax, void* gdir, int nthreads) {
    emu::launch(gx / WORKGROUP_X, gy / WORKGROUP_Y, WORKGROUP_X, WORKGROUP_Y, [&]() {
        calculateScore((GlobalMatrix*)m, x, y, nb, s, t, (GlobalMaxima*)gmax, (GlobalDirection*)gdir); },
        nthreads);
}
extern "C" void emu_calculateScoreAffineGap(unsigned gx, unsigned gy, void* m, void* mi, void* mj,
        unsigned x, unsigned y, unsigned nb, char* s, char* t, void* gmax, void* gdir, int nthreads) {
    emu::launch(gx / WORKGROUP_X, gy / WORKGROUP_Y, WORKGROUP_X, WORKGROUP_Y, [&]() {
        calculateScoreAffineGap((GlobalMatrix*)m, (GlobalMatrix*)mi, (GlobalMatrix*)mj, x, y, nb, s, t,
                                (GlobalMaxima*)gmax, (GlobalDirection*)gdir); }, nthreads);
}
extern "C" void emu_traceback(unsigned gx, unsigned gy, void* m, unsigned x, unsigned y, unsigned nb,
        void* gmax, void* gdir, unsigned* idx, void* sp, float* mps, void* sem, int nthreads) {
    emu::launch(gx / WORKGROUP_X, gy / WORKGROUP_Y, WORKGROUP_X, WORKGROUP_Y, [&]() {
        traceback((GlobalMatrix*)m, x, y, nb, (GlobalMaxima*)gmax, (GlobalDirection*)gdir, idx,
                  (StartingPoints*)sp, mps, (GlobalSemaphores*)sem); }, nthreads);
}
extern "C" void emu_tracebackAffineGap(unsigned gx, unsigned gy, void* m, void* mi, void* mj,
        unsigned x, unsigned y, unsigned nb, void* gmax, void* gdir, unsigned* idx, void* sp,
        float* mps, void* sem, int nthreads) {
    emu::launch(gx / WORKGROUP_X, gy / WORKGROUP_Y, WORKGROUP_X, WORKGROUP_Y, [&]() {
        tracebackAffineGap((GlobalMatrix*)m, (GlobalMatrix*)mi, (GlobalMatrix*)mj, x, y, nb,
                           (GlobalMaxima*)gmax, (GlobalDirection*)gdir, idx, (StartingPoints*)sp, mps,
                           (GlobalSemaphores*)sem); }, nthreads);
}
"""


# The reference host driver's launch loops (SmithWaterman._calculate_score,
# SmithWaterman.py:591-618, and _traceback_host, :626-655) over the OpenCL CPU
# kernels, with SmithWatermanCPU's launch shapes (SmithWatermanOcl.py:459-511):
# one call runs a whole batch.
_OCL_CPU_LOOPS = r"""
extern "C" void emu_run_cpu_path(void* m, void* mi, void* mj, char* s, char* t, void* gmax, void* gdir,
        unsigned* idx_inc, void* sp, float* mps, void* sem, int affine, int nthreads) {
    const int xd = XdivSHARED_X, yd = YdivSHARED_Y;
    const int maxb = xd < yd ? xd : yd, dec = xd + yd - maxb;
    int idx = 0, idy = 0;
    for (int i = 1; i < xd + yd; ++i) {
        const int nb = i <= maxb ? i : (i >= dec ? xd + yd - i : maxb);
        const unsigned gx = NUMBER_SEQUENCES * WORKGROUP_X, gy = NUMBER_TARGETS * nb * WORKGROUP_Y;
        if (affine) emu_calculateScoreAffineGap(gx, gy, m, mi, mj, idx, idy, nb, s, t, gmax, gdir, nthreads);
        else emu_calculateScore(gx, gy, m, idx, idy, nb, s, t, gmax, gdir, nthreads);
        if (idx == xd - 1) ++idy;
        if (idx < xd - 1) ++idx;
    }
    idx = xd - 1;
    idy = yd - 1;
    for (int i = 1; i < xd + yd; ++i) {
        const int nb = i <= maxb ? i : (i >= dec ? xd + yd - i : maxb);
        const unsigned gx = NUMBER_SEQUENCES * WORKGROUP_X, gy = NUMBER_TARGETS * nb * WORKGROUP_Y;
        if (affine) emu_tracebackAffineGap(gx, gy, m, mi, mj, idx, idy, nb, gmax, gdir, idx_inc, sp, mps, sem,
                                           nthreads);
        else emu_traceback(gx, gy, m, idx, idy, nb, gmax, gdir, idx_inc, sp, mps, sem, nthreads);
        if (idy == 0) --idx;
        if (idy > 0) --idy;
    }
}
"""


def _import_reference_codegen():
    if REFERENCE_ROOT not in sys.path:
        sys.path.insert(0, REFERENCE_ROOT)
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        from pyPaSWAS.Core import PaSWAS  # reference template code (PaSWAS.py:5-144)
    return PaSWAS


def expand_source(score, n_sequences, n_targets, x, y, flavour="cuda"):
    """Template-expand the reference kernel source exactly as the reference does
    (SmithWatermanCuda.py:28-33,170-174 for CUDA; SmithWatermanOcl.py:46-51 and
    PaSWAS.CPUcode for the OpenCL CPU device)."""
    PaSWAS = _import_reference_codegen()
    logger = logging.getLogger("paswas_ref_codegen")
    if flavour == "cuda":
        code = PaSWAS.Cudacode(logger)
        code.set_shared_xy_code(8, 8)
    elif flavour == "ocl_cpu":
        code = PaSWAS.CPUcode(logger)
        code.set_shared_xy_code(8, 8, 4, 4)
    else:
        raise ValueError(flavour)
    code.set_direction_code(NO_DIRECTION, UPPER_LEFT, UPPER, LEFT, STOP)
    return code.get_code(score, n_sequences, n_targets, x, y)


def build(score, n_sequences, n_targets, x, y, flavour="cuda", out_dir=OUT_DIR):
    """Returns the path of the emulated reference kernel library for this shape."""
    src = expand_source(score, n_sequences, n_targets, x, y, flavour)
    src += _CUDA_LAUNCHERS if flavour == "cuda" else _OCL_CPU_LAUNCHERS + _OCL_CPU_LOOPS
    with open(os.path.join(HERE, "kernel_emu.hpp")) as f:
        shim = f.read()
    tag = hashlib.sha1((flavour + shim + src).encode()).hexdigest()[:16]
    os.makedirs(out_dir, exist_ok=True)
    so_path = os.path.join(out_dir, "ref_%s_%s.so" % (flavour, tag))
    if os.path.exists(so_path):
        return so_path
    cpp_path = os.path.join(out_dir, "ref_%s_%s.cpp" % (flavour, tag))
    with open(cpp_path, "w") as f:
        f.write('#include "kernel_emu.hpp"\n')
        f.write(src)
    stub_inc = os.path.join(HERE, "stub_include")
    cmd = ["g++", "-std=c++17", "-O2", "-ffp-contract=off", "-fno-fast-math", "-shared", "-fPIC",
           "-w", "-I", HERE, "-I", stub_inc, "-o", so_path + ".tmp", cpp_path, "-lpthread"]
    subprocess.run(cmd, check=True)
    os.replace(so_path + ".tmp", so_path)
    return so_path
