"""The C ABI called from plain C, as a Fortran program binds it: the harness
tests/c_harness/cirsrtfg_harness.c keeps the layer, path and gradient arrays
in static arrays with the reference's leading dimensions (MAXLAY, MAXV,
MAXGAS+2+MAXCON, MAXPRO) and passes ld_* = 0.  No Python on its call path.

CPU: the header compiles as C11 and the harness links against the library;
without a GPU the library refuses to create a context (exit status 3).
GPU: its outputs are bit-identical to the same job called through the
Python binding with compact arrays."""
import os
import subprocess
import tempfile

import numpy as np
import pytest

from radtrancode_b200 import _lib, synth

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
SRC = os.path.join(HERE, "c_harness", "cirsrtfg_harness.c")


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def build_harness(out_dir):
    lib = _lib.build()
    exe = os.path.join(out_dir, "cirsrtfg_harness")
    libdir = os.path.dirname(lib)
    subprocess.run(["gcc", "-O2", "-Wall", "-Wextra", "-Werror", "-std=c11", "-I", os.path.join(ROOT, "include"),
                    "-o", exe, SRC, "-L", libdir, "-lradtran_b200", f"-Wl,-rpath,{libdir}"], check=True)
    return exe


def dump_inputs(path, kt, cia, job):
    """The harness's input file (layout in cirsrtfg_harness.c)."""
    L, G, P = job.nlayer, job.ngas, job.npath
    i32 = lambda *v: np.array(v, np.int32).tobytes()
    f32 = lambda a: np.ascontiguousarray(a, np.float32).tobytes()
    with open(path, "wb") as f:
        f.write(i32(kt.ntab, kt.np_, kt.nt, kt.ng))
        for a in (kt.lnp, kt.tk, kt.delg, kt.vmin, kt.delv):
            f.write(f32(a))
        f.write(np.asarray(kt.nbin, np.int32).tobytes())
        f.write(f32(kt.data))
        f.write(f32([cia.dnu]))
        f.write(np.asarray(cia.temps, np.float64).tobytes())
        f.write(f32(cia.kcia))
        f.write(i32(L, G, P, job.npro, job.nv, job.nwave, len(job.vem), job.inormal, job.iray, job.itype,
                    job.ispace))
        f.write(f32([job.tsurf]))
        for a in (job.press, job.temp, job.delh):
            f.write(f32(a[:L]))
        for a in (job.pp, job.amount):
            for g in range(G):
                f.write(f32(a[:L, g]))
        for a in (job.idgas, job.isogas, job.ktab):
            f.write(np.asarray(a, np.int32).tobytes())
        f.write(np.asarray(job.nlayin, np.int32).tobytes())
        f.write(np.asarray(job.imod, np.int32).tobytes())
        for p in range(P):
            f.write(np.asarray(job.layinc[:L, p], np.int32).tobytes())
        for a in (job.scale, job.emtemp):
            for p in range(P):
                f.write(f32(a[:L, p]))
        for a in (job.dte, job.dam):
            for k in range(job.npro):
                f.write(f32(a[:L, k]))
        for k in range(job.npro):
            for q in range(G + 1):
                f.write(f32(job.xmap[:job.nv, q, k]))
        f.write(f32(job.vwave))
        f.write(f32(job.vem))
        f.write(f32(job.emissivity))


def test_c_harness_builds_and_refuses_without_gpu():
    with tempfile.TemporaryDirectory() as d:
        exe = build_harness(d)
        kt, cia, job = synth.config2(nwave=2, nlayer=10, nbin=2)
        dump_inputs(os.path.join(d, "in.bin"), kt, cia, job)
        r = subprocess.run([exe, os.path.join(d, "in.bin"), os.path.join(d, "out.bin")], capture_output=True)
        assert r.returncode == (0 if _has_gpu() else 3), r.stderr


@pytest.mark.gpu
def test_c_harness_matches_python_binding(ctx):
    kt, cia, job = synth.config2(nwave=16, nlayer=60, nbin=16)
    ctx.set_ktables(kt)
    ctx.set_cia(cia)
    c, g, gt = ctx.cirsrtfg_wave(job)
    with tempfile.TemporaryDirectory() as d:
        exe = build_harness(d)
        dump_inputs(os.path.join(d, "in.bin"), kt, cia, job)
        r = subprocess.run([exe, os.path.join(d, "in.bin"), os.path.join(d, "out.bin")], capture_output=True)
        assert r.returncode == 0, r.stderr
        out = np.fromfile(os.path.join(d, "out.bin"), np.float32)
    n1 = job.npath * job.nwave
    assert out.size == 2 * n1 + n1 * job.nv
    assert np.array_equal(out[:n1], c)
    assert np.array_equal(out[n1:n1 + n1 * job.nv], g)
    assert np.array_equal(out[n1 + n1 * job.nv:], gt)
