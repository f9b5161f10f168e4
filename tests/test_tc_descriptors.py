"""The tensor-core GEMM's descriptors (the-solver_b200/csrc/tc_gemm.cuh) against
CUTLASS's own definitions of the Blackwell UMMA bitfields
(cute/arch/mma_sm100_desc.hpp: SmemDescriptor, InstrDescriptor), on the host: the
shared-memory descriptor of the canonical K-major layout without swizzle (version 1,
leading byte offset = the K-adjacent core matrix, stride byte offset = the next 8-row
block), the kind::f16 instruction descriptor for bf16 x bf16 -> fp32 at M = 128,
N = 64 and 128, and the element offsets of the staged tiles against CuTe's stated
canonical form ((8, m), (8, 2)) : ((8, SBO), (1, LBO)); and for the weight-gradient
kernel's MN-major operands, the descriptor that CuTe's own make_umma_desc<Major::MN>
derives from the layout ((8, MN/8), (8, 2)) : ((1, 64), (8, LBO/2)) (elements), the
element offsets of that layout, and the instruction descriptor with both major bits.
Uses the CUTLASS headers vendored with flashinfer; skips where they or nvcc are absent."""
import importlib.util
import os
import shutil
import subprocess

import pytest

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))

SOURCE = r"""
#include <cstdio>
#include <cute/tensor.hpp>
#include <cute/atom/mma_traits_sm100.hpp>
#include "tc_gemm.cuh"
template <int MN, int LBOE>
int check_mn() {
    using namespace cute;
    int bad = 0;
    auto L = make_layout(make_shape(make_shape(_8{}, Int<MN / 8>{}), make_shape(_8{}, _2{})),
                         make_stride(make_stride(_1{}, _64{}), make_stride(_8{}, Int<LBOE>{})));
    auto t = make_tensor(make_smem_ptr(reinterpret_cast<cutlass::bfloat16_t*>(0)), L);
    UMMA::SmemDescriptor d = UMMA::make_umma_desc<UMMA::Major::MN>(t);
    d.start_address_ = 0;
    if (uint64_t(d) != b200::tc::smem_desc(0, LBOE * 2, 128)) ++bad;
    for (int mn = 0; mn < MN; ++mn) for (int k = 0; k < 16; ++k)
        if (unsigned(L(mn, k)) * 2 != b200::tc::mnmajor_offset<MN>(mn, k)) ++bad;
    return bad;
}
int main() {
    int bad = check_mn<128, 1024>() + check_mn<64, 512>();
    {
        cute::UMMA::InstrDescriptor i;
        i.desc_ = 0;
        i.c_format_ = 1;
        i.a_format_ = uint8_t(cute::UMMA::F16F32Format::BF16);
        i.b_format_ = uint8_t(cute::UMMA::F16F32Format::BF16);
        i.a_major_ = 1; i.b_major_ = 1; i.n_dim_ = 64 >> 3; i.m_dim_ = 128 >> 4;
        if (uint32_t(i) != b200::tc::instr_desc_bf16_mn(128, 64)) ++bad;
    }
    const unsigned addrs[] = {0u, 1024u, 49152u, 65792u};
    const unsigned Ks[] = {16u, 64u, 128u};
    for (unsigned a : addrs) for (unsigned K : Ks) {
        cute::UMMA::SmemDescriptor d;
        d.start_address_ = a >> 4;
        d.leading_byte_offset_ = 128 >> 4;
        d.stride_byte_offset_ = (K / 8 * 128) >> 4;
        d.version_ = 1;
        d.base_offset_ = 0;
        d.lbo_mode_ = 0;
        d.layout_type_ = uint8_t(cute::UMMA::LayoutType::SWIZZLE_NONE);
        if (uint64_t(d) != b200::tc::smem_desc(a, 128, K / 8 * 128)) ++bad;
    }
    for (int N : {64, 128}) {
        cute::UMMA::InstrDescriptor i;
        i.desc_ = 0;
        i.c_format_ = 1;
        i.a_format_ = uint8_t(cute::UMMA::F16F32Format::BF16);
        i.b_format_ = uint8_t(cute::UMMA::F16F32Format::BF16);
        i.a_major_ = 0; i.b_major_ = 0; i.n_dim_ = N >> 3; i.m_dim_ = 128 >> 4;
        if (uint32_t(i) != b200::tc::instr_desc_bf16(128, N)) ++bad;
    }
    for (int K : {16, 64, 128}) for (int r = 0; r < 128; ++r) for (int k = 0; k < K; ++k) {
        const unsigned expect = unsigned(((r / 8) * (K / 8 * 64) + (r % 8) * 8 + (k / 8) * 64 + (k % 8)) * 2);
        const unsigned got = K == 16 ? b200::tc::kmajor_offset<16>(r, k)
                           : K == 64 ? b200::tc::kmajor_offset<64>(r, k) : b200::tc::kmajor_offset<128>(r, k);
        if (expect != got) ++bad;
    }
    printf("mismatches %d\n", bad);
    return bad != 0;
}
"""


def _cutlass_include():
    spec = importlib.util.find_spec("flashinfer")
    if spec is None or not spec.submodule_search_locations:
        return None
    for loc in spec.submodule_search_locations:
        path = os.path.join(loc, "data", "cutlass", "include")
        if os.path.isfile(os.path.join(path, "cute", "arch", "mma_sm100_desc.hpp")):
            return path
    return None


def test_descriptors_match_cutlass(tmp_path):
    inc = _cutlass_include()
    if inc is None or shutil.which("nvcc") is None:
        pytest.skip("CUTLASS headers or nvcc absent")
    src = tmp_path / "chk.cu"
    src.write_text(SOURCE)
    exe = tmp_path / "chk"
    r = subprocess.run(["nvcc", "-std=c++17", "-I" + inc, "-I" + os.path.join(ROOT, "the-solver_b200", "csrc"),
                        str(src), "-o", str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
    out = subprocess.run([str(exe)], capture_output=True, text=True)
    assert out.returncode == 0 and "mismatches 0" in out.stdout, out.stdout
