"""Host logic of the shared-memory transforms (no GPU): the radix plans of the
specialised sizes, the digit-reversed output order the preconditioner
multiplies in, and the per-stage twiddle tables the stages index.

A small host program built with nvcc from ``nsrno_b200/csrc/nsr_common.cuh``
prints the plan functions' results; a numpy restatement of the same
decimation-in-frequency stages checks them."""
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

from conftest import ROOT

SIZES = [8, 24, 48, 64, 81, 96, 162, 256, 384, 512, 768, 1024, 1536, 2048,
         35, 110, 770, 961, 1056, 1121, 1216, 1210, 2 * 61]


def _smooth(n):
    """True for n = 2^a 3^b."""
    for p in (2, 3):
        while n % p == 0:
            n //= p
    return n == 1


SMOOTH = [n for n in SIZES if _smooth(n)]

PROBE = r"""
#include <cstdio>
#include "nsr_common.cuh"
int main() {
  const int sizes[] = {%s};
  for (int n : sizes) {
    int radix[NSR_MAX_RADIX_STAGES], nst = 0;
    if (!nsr_make_radices(n, radix, &nst)) { std::printf("bad %%d\n", n); continue; }
    std::printf("n %%d", n);
    std::printf(" radix");
    for (int s = 0; s < nst; ++s) std::printf(" %%d", radix[s]);
    std::printf(" offset");
    for (int s = 0; s < nst; ++s) std::printf(" %%d", nsr_twiddle_offset(n, nsr_stage_len(n, s)));
    std::printf(" total %%d", nsr_twiddle_offset(n, 0));
    std::printf(" rev");
    for (int p = 0; p < n; ++p) std::printf(" %%d", nsr_digit_reverse(p, n, radix, nst));
    std::printf("\n");
  }
  return 0;
}
""" % ", ".join(str(n) for n in SIZES)


@pytest.fixture(scope="module")
def plans(tmp_path_factory):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(nvcc).exists():
        pytest.skip("nvcc not available")
    d = tmp_path_factory.mktemp("fftplan")
    src, exe = d / "probe.cu", d / "probe"
    src.write_text(PROBE)
    subprocess.run([nvcc, "-std=c++17", f"-I{ROOT / 'include'}", f"-I{ROOT / 'nsrno_b200' / 'csrc'}",
                    str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    plans = {}
    for line in out.splitlines():
        tok = line.split()
        assert tok[0] == "n", line
        n = int(tok[1])
        i_r, i_o, i_t, i_v = tok.index("radix"), tok.index("offset"), tok.index("total"), tok.index("rev")
        plans[n] = dict(radix=[int(t) for t in tok[i_r + 1:i_o]], offset=[int(t) for t in tok[i_o + 1:i_t]],
                        total=int(tok[i_t + 1]), rev=np.array([int(t) for t in tok[i_v + 1:]]))
    return plans


def dif_forward(x, radix):
    """The forward stages as the kernels run them: stage s of length L and
    radix R takes, for block o and butterfly j < m = L/R, the elements
    o L + j + q m (q < R), applies the length-R DFT and multiplies output k by
    exp(-2 pi i j k / L), storing output k at o L + j + k m."""
    y = np.array(x, dtype=np.complex128)
    n, L = y.size, y.size
    for R in radix:
        m = L // R
        F = np.exp(-2j * np.pi * np.outer(np.arange(R), np.arange(R)) / R)
        for o in range(n // L):
            for j in range(m):
                idx = o * L + j + m * np.arange(R)
                v = F @ y[idx]
                y[idx] = v * np.exp(-2j * np.pi * j * np.arange(R) / L)
        L = m
    return y


def test_every_size_has_a_plan(plans):
    assert sorted(plans) == sorted(SIZES)
    primes = {q for q in range(5, 62) if all(q % r for r in range(2, q))}
    for n, p in plans.items():
        assert int(np.prod(p["radix"])) == n
        assert set(p["radix"]) <= {2, 3, 4, 8, 16} | primes
        if n in SMOOTH:   # 2^a 3^b: the power-of-two and radix-3 stages only
            assert set(p["radix"]) <= {2, 3, 4, 8, 16}


def test_sizes_with_a_prime_factor_above_61_have_no_plan(tmp_path):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(nvcc).exists():
        pytest.skip("nvcc not available")
    src, exe = tmp_path / "bad.cu", tmp_path / "bad"
    src.write_text('#include <cstdio>\n#include "nsr_common.cuh"\nint main() { int r[NSR_MAX_RADIX_STAGES], k;'
                   ' std::printf("%d %d %d %d\\n", nsr_make_radices(134, r, &k), nsr_make_radices(2 * 1021, r, &k),'
                   ' nsr_make_radices(4096, r, &k), nsr_make_radices(122, r, &k)); return 0; }\n')
    subprocess.run([nvcc, "-std=c++17", f"-I{ROOT / 'include'}", f"-I{ROOT / 'nsrno_b200' / 'csrc'}",
                    str(src), "-o", str(exe)], check=True)
    assert subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split() == \
        ["0", "0", "0", "1"]


def test_sizes_divisible_by_16_end_with_a_radix_16_stage(plans):
    # the fused column stage and the padded row layout rely on it
    for n, p in plans.items():
        if n % 16 == 0:
            assert p["radix"][-1] == 16, n


def test_digit_reversed_order_matches_the_stages(plans):
    rng = np.random.default_rng(0)
    for n, p in plans.items():
        rev = p["rev"]
        assert sorted(rev.tolist()) == list(range(n))
        x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
        y = dif_forward(x, p["radix"])
        assert np.max(np.abs(y - np.fft.fft(x)[rev])) < 1e-9 * n


def test_stage_twiddle_tables_are_sized_as_the_stages_index_them(plans):
    # stage s (length L, radix R, m = L/R > 1) owns (R-1) m entries, entry
    # (k-1) m + j for 1 <= k < R, j < m; the stage with m == 1 owns none
    for n, p in plans.items():
        L, off = n, 0
        for s, R in enumerate(p["radix"]):
            m = L // R
            assert p["offset"][s] == off, (n, s)
            if m > 1:
                off += (R - 1) * m
            L = m
        assert p["total"] == off
        assert off < 2 * n
