// Generated by gen_roots128.py -- do not edit.
// w_128^m = exp(-2*pi*i*m/128) = (cos, -sin)(2*pi*m/128), m = 0..31,
// each part correctly rounded to double and to float.  Constant memory with
// static initialisers (internal linkage: every translation unit that includes
// this header holds its own copy, loaded with the module), so a loop index
// known after unrolling becomes a constant-bank operand.
#pragma once

namespace mb {
namespace roots128 {

constexpr int kCount = 32;
static __constant__ double kReD[kCount] = {
    0x1.0000000000000p+0, 0x1.ff621e3796d7ep-1, 0x1.fd88da3d12526p-1, 0x1.fa7557f08a517p-1,
    0x1.f6297cff75cb0p-1, 0x1.f0a7efb9230d7p-1, 0x1.e9f4156c62ddap-1, 0x1.e212104f686e5p-1,
    0x1.d906bcf328d46p-1, 0x1.ced7af43cc773p-1, 0x1.c38b2f180bdb1p-1, 0x1.b728345196e3ep-1,
    0x1.a9b66290ea1a3p-1, 0x1.9b3e047f38741p-1, 0x1.8bc806b151741p-1, 0x1.7b5df226aafafp-1,
    0x1.6a09e667f3bcdp-1, 0x1.57d69348ceca0p-1, 0x1.44cf325091dd6p-1, 0x1.30ff7fce17035p-1,
    0x1.1c73b39ae68c8p-1, 0x1.073879922ffeep-1, 0x1.e2b5d3806f63bp-2, 0x1.b5d1009e15cc0p-2,
    0x1.87de2a6aea963p-2, 0x1.58f9a75ab1fddp-2, 0x1.294062ed59f06p-2, 0x1.f19f97b215f1bp-3,
    0x1.8f8b83c69a60bp-3, 0x1.2c8106e8e613ap-3, 0x1.917a6bc29b42cp-4, 0x1.91f65f10dd814p-5};
static __constant__ double kImD[kCount] = {
    0.0, -0x1.91f65f10dd814p-5, -0x1.917a6bc29b42cp-4, -0x1.2c8106e8e613ap-3,
    -0x1.8f8b83c69a60bp-3, -0x1.f19f97b215f1bp-3, -0x1.294062ed59f06p-2, -0x1.58f9a75ab1fddp-2,
    -0x1.87de2a6aea963p-2, -0x1.b5d1009e15cc0p-2, -0x1.e2b5d3806f63bp-2, -0x1.073879922ffeep-1,
    -0x1.1c73b39ae68c8p-1, -0x1.30ff7fce17035p-1, -0x1.44cf325091dd6p-1, -0x1.57d69348ceca0p-1,
    -0x1.6a09e667f3bcdp-1, -0x1.7b5df226aafafp-1, -0x1.8bc806b151741p-1, -0x1.9b3e047f38741p-1,
    -0x1.a9b66290ea1a3p-1, -0x1.b728345196e3ep-1, -0x1.c38b2f180bdb1p-1, -0x1.ced7af43cc773p-1,
    -0x1.d906bcf328d46p-1, -0x1.e212104f686e5p-1, -0x1.e9f4156c62ddap-1, -0x1.f0a7efb9230d7p-1,
    -0x1.f6297cff75cb0p-1, -0x1.fa7557f08a517p-1, -0x1.fd88da3d12526p-1, -0x1.ff621e3796d7ep-1};
static __constant__ float kReF[kCount] = {
    0x1.0000000000000p+0f, 0x1.ff621e0000000p-1f, 0x1.fd88da0000000p-1f, 0x1.fa75580000000p-1f,
    0x1.f6297c0000000p-1f, 0x1.f0a7f00000000p-1f, 0x1.e9f4160000000p-1f, 0x1.e212100000000p-1f,
    0x1.d906bc0000000p-1f, 0x1.ced7b00000000p-1f, 0x1.c38b300000000p-1f, 0x1.b728340000000p-1f,
    0x1.a9b6620000000p-1f, 0x1.9b3e040000000p-1f, 0x1.8bc8060000000p-1f, 0x1.7b5df20000000p-1f,
    0x1.6a09e60000000p-1f, 0x1.57d6940000000p-1f, 0x1.44cf320000000p-1f, 0x1.30ff800000000p-1f,
    0x1.1c73b40000000p-1f, 0x1.07387a0000000p-1f, 0x1.e2b5d40000000p-2f, 0x1.b5d1000000000p-2f,
    0x1.87de2a0000000p-2f, 0x1.58f9a80000000p-2f, 0x1.2940620000000p-2f, 0x1.f19f980000000p-3f,
    0x1.8f8b840000000p-3f, 0x1.2c81060000000p-3f, 0x1.917a6c0000000p-4f, 0x1.91f6600000000p-5f};
static __constant__ float kImF[kCount] = {
    0.0f, -0x1.91f6600000000p-5f, -0x1.917a6c0000000p-4f, -0x1.2c81060000000p-3f,
    -0x1.8f8b840000000p-3f, -0x1.f19f980000000p-3f, -0x1.2940620000000p-2f, -0x1.58f9a80000000p-2f,
    -0x1.87de2a0000000p-2f, -0x1.b5d1000000000p-2f, -0x1.e2b5d40000000p-2f, -0x1.07387a0000000p-1f,
    -0x1.1c73b40000000p-1f, -0x1.30ff800000000p-1f, -0x1.44cf320000000p-1f, -0x1.57d6940000000p-1f,
    -0x1.6a09e60000000p-1f, -0x1.7b5df20000000p-1f, -0x1.8bc8060000000p-1f, -0x1.9b3e040000000p-1f,
    -0x1.a9b6620000000p-1f, -0x1.b728340000000p-1f, -0x1.c38b300000000p-1f, -0x1.ced7b00000000p-1f,
    -0x1.d906bc0000000p-1f, -0x1.e212100000000p-1f, -0x1.e9f4160000000p-1f, -0x1.f0a7f00000000p-1f,
    -0x1.f6297c0000000p-1f, -0x1.fa75580000000p-1f, -0x1.fd88da0000000p-1f, -0x1.ff621e0000000p-1f};

}  // namespace roots128
}  // namespace mb
