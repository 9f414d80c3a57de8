"""Resource guards for the hot kernels, read from ptxas's report (-Xptxas -v)
of the library's own sources, compiled for sm_100a on the host.

Two regressions of this kind were measured on the GPU: constraint code
compiled into the ODE kernels pushed the one-cell-per-thread kernel's
cell-claim lambda out of line (a 2.8 KB stack frame, 12 % slower) and raised
the plain forcing and Jacobian kernels from 32 to 80-116 registers (21 %
slower).  These tests fail if either comes back."""
import os
import re
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "micm_b200", "csrc")
FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-std=c++17", "-fmad=false",
         "--expt-relaxed-constexpr", "-Xptxas", "-v", "-c"]

pytestmark = pytest.mark.skipif(shutil.which("nvcc") is None, reason="nvcc not available")


def _parse(report):
    """{mangled name: {"stack": bytes, "spill_st": bytes, "spill_ld": bytes, "regs": n}}"""
    out, entry, props = {}, None, None
    for line in report.splitlines():
        m = re.search(r"Compiling entry function '([^']+)'", line)
        if m:
            entry = m.group(1)
            continue
        m = re.search(r"Function properties for (\S+)", line)
        if m:
            props = m.group(1)
            continue
        m = re.search(r"(\d+) bytes stack frame, (\d+) bytes spill stores, (\d+) bytes spill loads", line)
        if m and props:
            out.setdefault(props, {}).update(stack=int(m.group(1)), spill_st=int(m.group(2)),
                                             spill_ld=int(m.group(3)))
            props = None
            continue
        m = re.search(r"Used (\d+) registers", line)
        if m and entry:
            out.setdefault(entry, {})["regs"] = int(m.group(1))
    return out


@pytest.fixture(scope="module")
def reports(tmp_path_factory):
    tmp = tmp_path_factory.mktemp("ptxas")
    procs = {}
    for src in ("fused_thread.cu", "plain.cu"):
        procs[src] = subprocess.Popen(["nvcc"] + FLAGS + [src, "-o", str(tmp / (src + ".o"))], cwd=CSRC,
                                      stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    out = {}
    for src, p in procs.items():
        text, _ = p.communicate(timeout=900)
        assert p.returncode == 0, text[-2000:]
        out[src] = _parse(text)
    return out


def _named(table, kernel, dae):
    tag = "ILb1E" if dae else "ILb0E"
    return {k: v for k, v in table.items() if re.search(kernel + r"(_r\d+)?" + tag, k)}


def test_thread_kernel_keeps_its_helpers_inline(reports):
    t = reports["fused_thread.cu"]
    ode = _named(t, "k_fused_thread", dae=False)
    assert len(ode) == 4, sorted(t)  # the 32-, 40-, 64- and 96-register builds
    for name, r in ode.items():
        assert r["stack"] <= 512, (name, r)
    # nothing of the kernel body outlined into a separate device function
    outlined = [k for k in t if "fused_thread_body" in k and "k_fused_thread" not in k]
    assert not outlined, outlined


def test_plain_ode_stage_kernels_stay_small(reports):
    p = reports["plain.cu"]
    for kernel in ("k_forcing0", "k_jacobian", "k_stage_forcing"):
        found = _named(p, kernel, dae=False)
        assert len(found) == 1, (kernel, sorted(p))
        (r,) = found.values()
        assert r["regs"] <= 48, (kernel, r)
