"""The tensor-core descriptor encodings of ggems_b200/csrc/gg_umma_desc.cuh
against CuTe's bitfield definitions of the same descriptors
(cute/arch/mma_sm100_desc.hpp: UMMA::SmemDescriptor, UMMA::InstrDescriptor):
a host program built with nvcc fills both for a sweep of addresses, offsets,
swizzles, tile shapes and majorness and compares the bits.  CPU only; skipped
where no CUTLASS / CuTe tree is installed (the build does not need one)."""

import importlib.util
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

HARNESS = r'''
#include <cstdio>
#include <cute/arch/mma_sm100_desc.hpp>
#include "gg_umma_desc.cuh"
int main() {
  int bad = 0, n = 0;
  const cute::UMMA::LayoutType lt[3] = {cute::UMMA::LayoutType::SWIZZLE_32B, cute::UMMA::LayoutType::SWIZZLE_64B,
                                        cute::UMMA::LayoutType::SWIZZLE_128B};
  const int rows[3] = {32, 64, 128};
  for (uint32_t addr = 0; addr < (1u << 18); addr += 1024 + 16)
    for (uint32_t lbo : {16u, 1024u, 8192u, 65520u})
      for (int s = 0; s < 3; ++s) {
        cute::UMMA::SmemDescriptor d;
        d.desc_ = 0;
        d.start_address_ = static_cast<uint16_t>(addr >> 4);
        d.leading_byte_offset_ = static_cast<uint16_t>(lbo >> 4);
        d.stride_byte_offset_ = static_cast<uint16_t>((8 * rows[s]) >> 4);
        d.version_ = 1;
        d.base_offset_ = 0;
        d.lbo_mode_ = 0;
        d.layout_type_ = static_cast<uint8_t>(lt[s]);
        bad += d.desc_ != gg::umma_smem_desc(addr, lbo, 8 * rows[s], gg::umma_row_swizzle(rows[s]));
        ++n;
      }
  for (int m : {64, 128, 256})
    for (int nt = 8; nt <= 256; nt += 8)
      for (int am = 0; am < 2; ++am)
        for (int bm = 0; bm < 2; ++bm) {
          cute::UMMA::InstrDescriptor id;
          id.desc_ = 0;
          id.c_format_ = 1;
          id.a_format_ = 1;
          id.b_format_ = 1;
          id.a_major_ = am;
          id.b_major_ = bm;
          id.n_dim_ = static_cast<uint16_t>(nt >> 3);
          id.m_dim_ = static_cast<uint16_t>(m >> 4);
          bad += id.desc_ != gg::umma_idesc_bf16_f32(m, nt, am, bm);
          ++n;
        }
  printf("%d %d\n", n, bad);
  return bad != 0;
}
'''


def _cute_include():
    for pkg, sub in (("flashinfer", ("data", "cutlass", "include")), ("tilelang", ("3rdparty", "cutlass", "include"))):
        spec = importlib.util.find_spec(pkg)
        if spec and spec.submodule_search_locations:
            path = os.path.join(spec.submodule_search_locations[0], *sub)
            if os.path.exists(os.path.join(path, "cute", "arch", "mma_sm100_desc.hpp")):
                return path
    env = os.environ.get("CUTLASS_DIR")
    if env and os.path.exists(os.path.join(env, "include", "cute", "arch", "mma_sm100_desc.hpp")):
        return os.path.join(env, "include")
    return None


def test_descriptors_match_cute(tmp_path):
    inc = _cute_include()
    if inc is None or shutil.which("nvcc") is None:
        pytest.skip("no CuTe tree or nvcc")
    (tmp_path / "h.cu").write_text(HARNESS)
    exe = tmp_path / "h"
    subprocess.check_call(["nvcc", "-std=c++17", "-I" + inc, "-I" + os.path.join(ROOT, "ggems_b200", "csrc"),
                           str(tmp_path / "h.cu"), "-o", str(exe)])
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    n, bad = map(int, out.stdout.split())
    print("descriptors compared: %d, different: %d" % (n, bad))
    assert out.returncode == 0 and bad == 0 and n > 1000
