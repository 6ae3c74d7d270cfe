// textio.cu -- the reference's ASCII result files, formatted on the GPU.
//
// The reference writes its results with fprintf: save_pressure / save_flux
// (posprocessing_output.c:200-296), save_pressure_1d / save_flux_1d
// (:437-661) and vts_StructuredGrid_file (vtk.c:8-76).  At 256^3 that is
// ~17M lines of four to six conversions each, seconds of single-threaded
// printf, longer than the solve.  Here every line is formatted by one GPU
// thread into a fixed-width slot, the slot lengths are prefix-summed, the
// text is compacted in HBM and copied out in chunks that overlap the file
// write.  The bytes are the ones glibc's printf writes for the same
// format strings: conversions are exact (the decimal digits of the binary
// value, rounded half to even, from 128-bit integer arithmetic), so the
// files are identical to the reference's.  A value the exact path does not
// cover (NaN, infinity, or a magnitude outside the exact range: for %1.9e
// below ~1e-77 or above ~1e36) sends its line to the host, which formats it
// with snprintf and the same format string.
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <string>
#include <vector>

#include "solver.cuh"
#include "../../include/hmfem_karst.h"
#include "../../include/hmfem_textio.h"

namespace hm {

namespace {

typedef unsigned __int128 u128;

__constant__ unsigned long long c_pow5[28] = {
    1ull, 5ull, 25ull, 125ull, 625ull, 3125ull, 15625ull, 78125ull, 390625ull,
    1953125ull, 9765625ull, 48828125ull, 244140625ull, 1220703125ull,
    6103515625ull, 30517578125ull, 152587890625ull, 762939453125ull,
    3814697265625ull, 19073486328125ull, 95367431640625ull, 476837158203125ull,
    2384185791015625ull, 11920928955078125ull, 59604644775390625ull,
    298023223876953125ull, 1490116119384765625ull, 7450580596923828125ull};

// 5^b, b = 0..86, as four little-endian 64-bit words (5^86 < 2^200)
__constant__ unsigned long long c_pow5w[87][4] = {
    {0x0000000000000001ull, 0x0000000000000000ull, 0x0000000000000000ull, 0x0000000000000000ull},
    {0x0000000000000005ull, 0x0000000000000000ull, 0x0000000000000000ull, 0x0000000000000000ull},
    {0x0000000000000019ull, 0x0000000000000000ull, 0x0000000000000000ull, 0x0000000000000000ull},
    {0x000000000000007dull, 0x0000000000000000ull, 0x0000000000000000ull, 0x0000000000000000ull},
    {0x0000000000000271ull, 0x0000000000000000ull, 0x0000000000000000ull, 0x0000000000000000ull},
    {0x0000000000000c35ull, 0x0000000000000000ull, 0x0000000000000000ull, 0x0000000000000000ull},
    {0x0000000000003d09ull, 0x0000000000000000ull, 0x0000000000000000ull, 0x0000000000000000ull},
    {0x000000000001312dull, 0x0000000000000000ull, 0x0000000000000000ull, 0x0000000000000000ull},
    {0x000000000005f5e1ull, 0x0000000000000000ull, 0x0000000000000000ull, 0x0000000000000000ull},
    {0x00000000001dcd65ull, 0x0000000000000000ull, 0x0000000000000000ull, 0x0000000000000000ull},
    {0x00000000009502f9ull, 0x0000000000000000ull, 0x0000000000000000ull, 0x0000000000000000ull},
    {0x0000000002e90eddull, 0x0000000000000000ull, 0x0000000000000000ull, 0x0000000000000000ull},
    {0x000000000e8d4a51ull, 0x0000000000000000ull, 0x0000000000000000ull, 0x0000000000000000ull},
    {0x0000000048c27395ull, 0x0000000000000000ull, 0x0000000000000000ull, 0x0000000000000000ull},
    {0x000000016bcc41e9ull, 0x0000000000000000ull, 0x0000000000000000ull, 0x0000000000000000ull},
    {0x000000071afd498dull, 0x0000000000000000ull, 0x0000000000000000ull, 0x0000000000000000ull},
    {0x0000002386f26fc1ull, 0x0000000000000000ull, 0x0000000000000000ull, 0x0000000000000000ull},
    {0x000000b1a2bc2ec5ull, 0x0000000000000000ull, 0x0000000000000000ull, 0x0000000000000000ull},
    {0x000003782dace9d9ull, 0x0000000000000000ull, 0x0000000000000000ull, 0x0000000000000000ull},
    {0x00001158e460913dull, 0x0000000000000000ull, 0x0000000000000000ull, 0x0000000000000000ull},
    {0x000056bc75e2d631ull, 0x0000000000000000ull, 0x0000000000000000ull, 0x0000000000000000ull},
    {0x0001b1ae4d6e2ef5ull, 0x0000000000000000ull, 0x0000000000000000ull, 0x0000000000000000ull},
    {0x000878678326eac9ull, 0x0000000000000000ull, 0x0000000000000000ull, 0x0000000000000000ull},
    {0x002a5a058fc295edull, 0x0000000000000000ull, 0x0000000000000000ull, 0x0000000000000000ull},
    {0x00d3c21bcecceda1ull, 0x0000000000000000ull, 0x0000000000000000ull, 0x0000000000000000ull},
    {0x0422ca8b0a00a425ull, 0x0000000000000000ull, 0x0000000000000000ull, 0x0000000000000000ull},
    {0x14adf4b7320334b9ull, 0x0000000000000000ull, 0x0000000000000000ull, 0x0000000000000000ull},
    {0x6765c793fa10079dull, 0x0000000000000000ull, 0x0000000000000000ull, 0x0000000000000000ull},
    {0x04fce5e3e2502611ull, 0x0000000000000002ull, 0x0000000000000000ull, 0x0000000000000000ull},
    {0x18f07d736b90be55ull, 0x000000000000000aull, 0x0000000000000000ull, 0x0000000000000000ull},
    {0x7cb2734119d3b7a9ull, 0x0000000000000032ull, 0x0000000000000000ull, 0x0000000000000000ull},
    {0x6f7c40458122964dull, 0x00000000000000fcull, 0x0000000000000000ull, 0x0000000000000000ull},
    {0x2d6d415b85acef81ull, 0x00000000000004eeull, 0x0000000000000000ull, 0x0000000000000000ull},
    {0xe32246c99c60ad85ull, 0x00000000000018a6ull, 0x0000000000000000ull, 0x0000000000000000ull},
    {0x6fab61f00de36399ull, 0x0000000000007b42ull, 0x0000000000000000ull, 0x0000000000000000ull},
    {0x2e58e9b04570f1fdull, 0x000000000002684cull, 0x0000000000000000ull, 0x0000000000000000ull},
    {0xe7bc90715b34b9f1ull, 0x00000000000c097cull, 0x0000000000000000ull, 0x0000000000000000ull},
    {0x86aed236c807a1b5ull, 0x00000000003c2f70ull, 0x0000000000000000ull, 0x0000000000000000ull},
    {0xa16a1b11e8262889ull, 0x00000000012ced32ull, 0x0000000000000000ull, 0x0000000000000000ull},
    {0x2712875988becaadull, 0x0000000005e0a1fdull, 0x0000000000000000ull, 0x0000000000000000ull},
    {0xc35ca4bfabb9f561ull, 0x000000001d6329f1ull, 0x0000000000000000ull, 0x0000000000000000ull},
    {0xd0cf37be5aa1cae5ull, 0x0000000092efd1b8ull, 0x0000000000000000ull, 0x0000000000000000ull},
    {0x140c16b7c528f679ull, 0x00000002deaf189cull, 0x0000000000000000ull, 0x0000000000000000ull},
    {0x643c7196d9ccd05dull, 0x0000000e596b7b0cull, 0x0000000000000000ull, 0x0000000000000000ull},
    {0xf52e37f2410011d1ull, 0x00000047bf19673dull, 0x0000000000000000ull, 0x0000000000000000ull},
    {0xc9e717bb45005915ull, 0x00000166bb7f0435ull, 0x0000000000000000ull, 0x0000000000000000ull},
    {0xf18376a85901bd69ull, 0x00000701a97b150cull, 0x0000000000000000ull, 0x0000000000000000ull},
    {0xb7915149bd08b30dull, 0x000023084f676940ull, 0x0000000000000000ull, 0x0000000000000000ull},
    {0x95d69670b12b7f41ull, 0x0000af298d050e43ull, 0x0000000000000000ull, 0x0000000000000000ull},
    {0xed30f03375d97c45ull, 0x00036bcfc1194751ull, 0x0000000000000000ull, 0x0000000000000000ull},
    {0xa1f4b1014d3f6d59ull, 0x00111b0ec57e6499ull, 0x0000000000000000ull, 0x0000000000000000ull},
    {0x29c77506823d22bdull, 0x00558749db77f700ull, 0x0000000000000000ull, 0x0000000000000000ull},
    {0xd0e549208b31adb1ull, 0x01aba4714957d300ull, 0x0000000000000000ull, 0x0000000000000000ull},
    {0x147a6da2b7f86475ull, 0x085a36366eb71f04ull, 0x0000000000000000ull, 0x0000000000000000ull},
    {0x6664242d97d9f649ull, 0x29c30f1029939b14ull, 0x0000000000000000ull, 0x0000000000000000ull},
    {0xfff4b4e3f741cf6dull, 0xd0cf4b50cfe20765ull, 0x0000000000000000ull, 0x0000000000000000ull},
    {0xffc78873d4490d21ull, 0x140c78940f6a24fdull, 0x0000000000000004ull, 0x0000000000000000ull},
    {0xfee5aa43256d41a5ull, 0x643e5ae44d12b8f5ull, 0x0000000000000014ull, 0x0000000000000000ull},
    {0xfa7c534fbb224839ull, 0xf537c675815d9ccdull, 0x0000000000000065ull, 0x0000000000000000ull},
    {0xe46da08ea7ab691dull, 0xca16e04b86d41005ull, 0x00000000000001fdull, 0x0000000000000000ull},
    {0x762422c946590d91ull, 0xf2726179a224501dull, 0x00000000000009f4ull, 0x0000000000000000ull},
    {0x4eb4adee5fbd43d5ull, 0xbc3be7602ab59093ull, 0x00000000000031c8ull, 0x0000000000000000ull},
    {0x898765a7deb25329ull, 0xad2b84e0d58bd2e0ull, 0x000000000000f8ebull, 0x0000000000000000ull},
    {0xafa4fc47597b9fcdull, 0x61d998642bbb1e62ull, 0x000000000004dc9aull, 0x0000000000000000ull},
    {0x6e38ed64bf6a1f01ull, 0xe93ff9f4daa797edull, 0x0000000000184f03ull, 0x0000000000000000ull},
    {0x271ca2f7bd129b05ull, 0x8e3fe1c84545f7a3ull, 0x0000000000798b13ull, 0x0000000000000000ull},
    {0xc38f2ed6b15d0719ull, 0xc73f68e95a5dd62full, 0x00000000025fb761ull, 0x0000000000000000ull},
    {0xd1cbea3176d1237dull, 0xe43d0c8ec3d52eeeull, 0x000000000bde94e8ull, 0x0000000000000000ull},
    {0x18fb92f75215b171ull, 0x75313ec9d329eaaaull, 0x000000003b58e88cull, 0x0000000000000000ull},
    {0x7ce9ded49a6c7735ull, 0x49f639f11fd19552ull, 0x0000000128bc8abeull, 0x0000000000000000ull},
    {0x70915a27041e5409ull, 0x71cf21b59f17ea9cull, 0x00000005cbaeb5b7ull, 0x0000000000000000ull},
    {0x32d6c2c31497a42dull, 0x390ba88c1b77950eull, 0x0000001cfa698c95ull, 0x0000000000000000ull},
    {0xfe31cdcf66f634e1ull, 0x1d3a4abc8955e946ull, 0x00000090e40fbeeaull, 0x0000000000000000ull},
    {0xf6f9050d02cf0865ull, 0x922375aeaead8e62ull, 0x000002d4744eba92ull, 0x0000000000000000ull},
    {0xd2dd19410e0b29f9ull, 0xdab14c696963c7eeull, 0x00000e264589a4dcull, 0x0000000000000000ull},
    {0x1e517e454637d1ddull, 0x45767e0f0ef2e7aaull, 0x000046bf5bb03850ull, 0x0000000000000000ull},
    {0x9797775a5f171951ull, 0x5b50764b4abe8652ull, 0x000161bcca711991ull, 0x0000000000000000ull},
    {0xf5f554c3db737e95ull, 0xc8924f7875b89f9cull, 0x0006e8aff4357fd6ull, 0x0000000000000000ull},
    {0xcdcaa7d3494178e9ull, 0xeadb8d5a4c9b1e10ull, 0x00228b6fc50b7f31ull, 0x0000000000000000ull},
    {0x04f547206e475c8dull, 0x9649c2c37f079654ull, 0x00acb92ed9397bf9ull, 0x0000000000000000ull},
    {0x18ca63a22764cec1ull, 0xef70cdd17b25efa4ull, 0x035f9dea3e1f6bdfull, 0x0000000000000000ull},
    {0x7bf3f22ac4f809c5ull, 0xad34051767bdae34ull, 0x10de1593369d1b5full, 0x0000000000000000ull},
    {0x6bc3bad5d8d830d9ull, 0x6204197506b46706ull, 0x54566be0111188deull, 0x0000000000000000ull},
    {0x1ad2a62d3c38f43dull, 0xea147f4921860320ull, 0xa5b01b605557ac57ull, 0x0000000000000001ull},
    {0x861d3ee22d1cc531ull, 0x92667c6da79e0fa0ull, 0x3c7088e1aab65db7ull, 0x0000000000000008ull},
    {0x9e923a6ae18fd9f5ull, 0xdc006e2446164e22ull, 0x2e32ac68558fd495ull, 0x0000000000000029ull},
    {0x18db241667cf41c9ull, 0x4c0226b55e6f86adull, 0xe6fd5e09abcf26edull, 0x00000000000000cdull}};

__constant__ unsigned long long c_pow10[20] = {
    1ull, 10ull, 100ull, 1000ull, 10000ull, 100000ull, 1000000ull, 10000000ull,
    100000000ull, 1000000000ull, 10000000000ull, 100000000000ull,
    1000000000000ull, 10000000000000ull, 100000000000000ull,
    1000000000000000ull, 10000000000000000ull, 100000000000000000ull,
    1000000000000000000ull, 10000000000000000000ull};

// |x| = m * 2^e2 with m < 2^53 (x finite, nonzero)
__device__ __forceinline__ void decompose(double x, unsigned long long &m, int &e2)
{
    const unsigned long long b = (unsigned long long)__double_as_longlong(x) & 0x7fffffffffffffffull;
    const int be = (int)(b >> 52);
    const unsigned long long f = b & ((1ull << 52) - 1);
    if (be == 0) { m = f; e2 = -1074; }
    else { m = f | (1ull << 52); e2 = be - 1075; }
}

// The q < 0 branch for 27 < b = -q <= 86 (small magnitudes): N0 = m 5^b
// held in four 64-bit words (< 2^253), then T = N0 >> sh with sh = -(e2 + b)
// and the remainder compared with 2^(sh-1) bit by bit.
__device__ bool wide_mul_pow5(unsigned long long m, int e2, int b, unsigned long long &T,
                              int &cmp)
{
    if (b > 86) return false;
    unsigned long long w[4];
    u128 carry = 0;
#pragma unroll
    for (int k = 0; k < 4; k++) {
        const u128 p = (u128)m * c_pow5w[b][k] + carry;
        w[k] = (unsigned long long)p;
        carry = p >> 64;
    }
    if (carry) return false;
    const int c = e2 + b;
    if (c >= 0) return false;  // a large value times 10^b: not reached for %e / %f here
    const int sh = -c;
    if (sh > 255) {  // the value is below 2^-2: T = 0, remainder below one half
        T = 0;
        cmp = -1;
        return true;
    }
    // T = bits [sh, sh + 64); nothing may be set above them
    auto bit = [&](int i) -> unsigned long long {
        return i < 0 || i > 255 ? 0ull : (w[i >> 6] >> (i & 63)) & 1ull;
    };
    auto word_at = [&](int i) -> unsigned long long {  // bits [i, i + 64)
        const int q0 = i >> 6, r0 = i & 63;
        unsigned long long lo = q0 < 4 ? w[q0] >> r0 : 0ull;
        unsigned long long hi = (r0 && q0 + 1 < 4) ? w[q0 + 1] << (64 - r0) : 0ull;
        return lo | hi;
    };
    for (int i = sh + 64; i < 256; i += 64)
        if (word_at(i) != 0ull) return false;
    T = word_at(sh);
    // remainder = bits [0, sh): compare with 2^(sh-1)
    bool low_nonzero = false;
    for (int i = 0; i < sh - 1; i += 64) {
        const int len = sh - 1 - i;
        unsigned long long v = word_at(i);
        if (len < 64) v &= (1ull << len) - 1;
        if (v) { low_nonzero = true; break; }
    }
    const unsigned long long top = bit(sh - 1);
    cmp = top ? (low_nonzero ? 1 : 0) : (low_nonzero ? -1 : -2);
    return true;
}

// T = floor(m 2^e2 / 10^q) and where the remainder lies: -2 zero, -1 below
// one half, 0 exactly one half, 1 above.  False when the operands leave the
// 128-bit range (or T leaves 64 bits).
__device__ bool div_pow10(unsigned long long m, int e2, int q, unsigned long long &T, int &cmp)
{
    if (q >= 0) {
        if (q > 27) return false;
        const int a = e2 - q;
        u128 N, Dn;
        if (a >= 0) {
            if (a > 74) return false;
            N = (u128)m << a;
            Dn = c_pow5[q];
        } else {
            if (-a > 64) return false;
            N = m;
            Dn = (u128)c_pow5[q] << (-a);
        }
        const u128 Tq = N / Dn, R = N - Tq * Dn;
        if (Tq >> 64) return false;
        T = (unsigned long long)Tq;
        const u128 R2 = R << 1;
        cmp = R == 0 ? -2 : (R2 < Dn ? -1 : (R2 == Dn ? 0 : 1));
        return true;
    }
    const int b = -q;
    if (b > 27) return wide_mul_pow5(m, e2, b, T, cmp);
    const u128 N0 = (u128)m * c_pow5[b];  // < 2^116
    const int c = e2 + b;
    if (c >= 0) {
        if (c > 11) return false;
        const u128 v = N0 << c;
        if (v >> 64) return false;
        T = (unsigned long long)v;
        cmp = -2;
        return true;
    }
    const int sh = -c;
    if (sh >= 127) {  // value below 2^-11: T = 0, remainder below one half
        T = 0;
        cmp = -1;
        return true;
    }
    const u128 Tq = N0 >> sh;
    const u128 R = N0 & (((u128)1 << sh) - 1), half = (u128)1 << (sh - 1);
    if (Tq >> 64) return false;
    T = (unsigned long long)Tq;
    cmp = R == 0 ? -2 : (R < half ? -1 : (R == half ? 0 : 1));
    return true;
}

__device__ __forceinline__ unsigned long long round_even(unsigned long long T, int cmp)
{
    return T + ((cmp == 1 || (cmp == 0 && (T & 1))) ? 1ull : 0ull);
}

// writes the n digits of v (zero-padded) at o; returns n
__device__ __forceinline__ int put_digits(char *o, unsigned long long v, int n)
{
    for (int i = n - 1; i >= 0; i--) {
        o[i] = (char)('0' + (int)(v % 10ull));
        v /= 10ull;
    }
    return n;
}

__device__ __forceinline__ int ndigits(unsigned long long v)
{
    int n = 1;
    while (n < 20 && v >= c_pow10[n]) n++;
    return n;
}

// printf("%.Pe", x); returns the length, or -1 (host formats it)
__device__ int fmt_e(double x, int P, char *o)
{
    if (isnan(x) || isinf(x) || P > 17) return -1;
    int n = 0;
    if (signbit(x)) o[n++] = '-';
    unsigned long long D = 0;
    int E = 0;
    if (x != 0.0) {
        unsigned long long m;
        int e2;
        decompose(x, m, e2);
        E = (int)floor(log10(fabs(x)));
        unsigned long long T = 0;
        int cmp = 0, tries = 0;
        for (;; tries++) {
            if (tries > 3 || !div_pow10(m, e2, E - P, T, cmp)) return -1;
            if (T < c_pow10[P]) { E--; continue; }
            if (P + 1 <= 19 && T >= c_pow10[P + 1]) { E++; continue; }
            break;
        }
        D = round_even(T, cmp);
        if (D == c_pow10[P + 1]) { D = c_pow10[P]; E++; }
    }
    // d.ddd...
    const unsigned long long lead = D / c_pow10[P];
    o[n++] = (char)('0' + (int)lead);
    if (P > 0) {
        o[n++] = '.';
        n += put_digits(o + n, D - lead * c_pow10[P], P);
    }
    o[n++] = 'e';
    o[n++] = E < 0 ? '-' : '+';
    const unsigned ae = (unsigned)(E < 0 ? -E : E);
    n += put_digits(o + n, ae, ae >= 100 ? 3 : 2);
    return n;
}

// printf("%.Nf", x); returns the length, or -1
__device__ int fmt_f(double x, int N, char *o)
{
    if (isnan(x) || isinf(x) || N > 17) return -1;
    int n = 0;
    if (signbit(x)) o[n++] = '-';
    unsigned long long D = 0;
    if (x != 0.0) {
        unsigned long long m, T;
        int e2, cmp;
        decompose(x, m, e2);
        if (!div_pow10(m, e2, -N, T, cmp)) return -1;
        D = round_even(T, cmp);
        if (D < T) return -1;  // wrapped past 2^64
    }
    const unsigned long long ip = D / c_pow10[N], fp = D - ip * c_pow10[N];
    n += put_digits(o + n, ip, ndigits(ip));
    if (N > 0) {
        o[n++] = '.';
        n += put_digits(o + n, fp, N);
    }
    return n;
}

__device__ __forceinline__ int put_str(char *o, const char *s)
{
    int n = 0;
    while (s[n]) { o[n] = s[n]; n++; }
    return n;
}

// ---- line layouts ------------------------------------------------------------

enum Layout {
    L_PRESSURE = 0,   // save_pressure: i, j, k order, blank lines
    L_FLUX = 1,       // save_flux
    L_VTS_VEL = 2,    // vts_StructuredGrid_file velocity block
    L_VTS_PRES = 3,   // ... pressure block
    L_VTS_POINTS = 4, // ... points block
    L_KARST_P = 5,    // save_pressure_1d, one conduit
    L_KARST_U = 6,    // save_flux_1d, one conduit
    L_NUM_E = 7,      // one "%.Pe\n" per value
    L_NUM_F = 8,      // one "%.Pf\n" per value
};

struct Job {
    int layout;
    long nrec;
    int nx, ny, nz;
    double hx, hy, hz;
    const double *p;
    const hmfem_ele *v;
    // conduit layouts: element i at (x0 + i dx, y0 + i dy, z0) ... (z0 + i dz)
    int x0, y0, z0, dx, dy, dz;
    const double *a, *b;  // pc[i][j] or ucr / ucl, element i at a[i * stride]
    int stride;
    int prec;
};

constexpr int kSlot = 192;  // bytes per line slot (longest line: ~150)

__device__ __forceinline__ double coord(double h, int i)
{
    return dmul(h, (double)i + 0.5);  // h.x*(i + 0.5)
}

// one line (record r of the job) at o; length or -1
__device__ int format_record(const Job &J, long r, char *o)
{
    int n = 0, w;
#define PUT(expr)              \
    do {                       \
        w = (expr);            \
        if (w < 0) return -1;  \
        n += w;                \
    } while (0)
    switch (J.layout) {
    case L_PRESSURE:
    case L_FLUX: {
        const long nyz = (long)J.ny * J.nz;
        const int i = (int)(r / nyz);
        const long rem = r - (long)i * nyz;
        const int j = (int)(rem / J.nz), k = (int)(rem - (long)j * J.nz);
        const long s = i + (long)J.nx * (j + (long)J.ny * k);
        PUT(fmt_f(coord(J.hx, i), 6, o + n)); o[n++] = ' ';
        PUT(fmt_f(coord(J.hy, j), 6, o + n)); o[n++] = ' ';
        PUT(fmt_f(coord(J.hz, k), 6, o + n)); o[n++] = ' ';
        if (J.layout == L_PRESSURE) {
            PUT(fmt_e(J.p[s], 9, o + n));
            o[n++] = '\n';
            if (k == J.nz - 1) {
                n += put_str(o + n, " \n");
                if (j == J.ny - 1) n += put_str(o + n, " \n");
            }
        } else {
            const hmfem_ele &e = J.v[s];
            PUT(fmt_e(dmul(0.5, dsub(e.r, e.l)), 9, o + n)); o[n++] = ' ';
            PUT(fmt_e(dmul(0.5, dsub(e.u, e.d)), 9, o + n)); o[n++] = ' ';
            PUT(fmt_e(dmul(0.5, dsub(e.t, e.b)), 9, o + n));
            n += put_str(o + n, " \n");
        }
        return n;
    }
    case L_VTS_VEL: {
        const hmfem_ele &e = J.v[r];
        PUT(fmt_e(dmul(0.5, dsub(e.r, e.l)), 8, o + n)); o[n++] = ' ';
        PUT(fmt_e(dmul(0.5, dsub(e.u, e.d)), 8, o + n)); o[n++] = ' ';
        PUT(fmt_e(dmul(0.5, dsub(e.t, e.b)), 8, o + n)); o[n++] = '\n';
        return n;
    }
    case L_VTS_PRES:
        PUT(fmt_e(J.p[r], 8, o + n)); o[n++] = '\n';
        return n;
    case L_VTS_POINTS: {
        const long nxy = (long)J.nx * J.ny;
        const int k = (int)(r / nxy);
        const long rem = r - (long)k * nxy;
        const int j = (int)(rem / J.nx), i = (int)(rem - (long)j * J.nx);
        PUT(fmt_f(coord(J.hx, i), 4, o + n)); o[n++] = ' ';
        PUT(fmt_f(coord(J.hy, j), 4, o + n)); o[n++] = ' ';
        PUT(fmt_f(coord(J.hz, k), 4, o + n));
        n += put_str(o + n, " \n");
        return n;
    }
    case L_KARST_P:
    case L_KARST_U: {
        const int i = (int)r;
        PUT(fmt_f(coord(J.hx, J.x0 + i * J.dx), 6, o + n)); o[n++] = ' ';
        PUT(fmt_f(coord(J.hy, J.y0 + i * J.dy), 6, o + n)); o[n++] = ' ';
        PUT(fmt_f(coord(J.hz, J.z0 + i * J.dz), 6, o + n)); o[n++] = ' ';
        const double val = J.layout == L_KARST_P
                               ? J.a[(long)i * J.stride]
                               : dmul(0.5, dsub(J.a[(long)i * J.stride], J.b[(long)i * J.stride]));
        PUT(fmt_e(val, 9, o + n)); o[n++] = '\n';
        return n;
    }
    case L_NUM_E:
        PUT(fmt_e(J.p[r], J.prec, o + n)); o[n++] = '\n';
        return n;
    case L_NUM_F:
        PUT(fmt_f(J.p[r], J.prec, o + n)); o[n++] = '\n';
        return n;
    }
#undef PUT
    return -1;
}

// records r0 .. r0 + m - 1 into slots; len = -1 marks a record for the host
__global__ void k_format(Job J, long r0, int m, char *__restrict__ slots, int *__restrict__ len,
                         int *nfall, int *fall, int fall_cap)
{
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < m; t += gridDim.x * blockDim.x) {
        __align__(16) char buf[kSlot];
        const int l = format_record(J, r0 + t, buf);
        if (l < 0) {
            len[t] = 0;
            const int q = atomicAdd(nfall, 1);
            if (q < fall_cap) fall[q] = t;
            continue;
        }
        // 16-byte stores into the slot (slots are 16-byte aligned)
        uint4 *o = (uint4 *)(slots + (long)t * kSlot);
        const uint4 *b = (const uint4 *)buf;
        for (int c = 0; c < (l + 15) / 16; c++) o[c] = b[c];
        len[t] = l;
    }
}

// text[off[t] ..] = slot t
__global__ void k_compact(int m, const char *__restrict__ slots, const int *__restrict__ len,
                          const int *__restrict__ off, char *__restrict__ text)
{
    // one warp per record: lanes copy the bytes
    const int lane = threadIdx.x & 31;
    const long w0 = (blockIdx.x * (long)blockDim.x + threadIdx.x) >> 5;
    const long nw = ((long)gridDim.x * blockDim.x) >> 5;
    for (long t = w0; t < m; t += nw) {
        const int l = len[t];
        const char *s = slots + t * kSlot;
        char *d = text + off[t];
        for (int c = lane; c < l; c += 32) d[c] = s[c];
    }
}

// ---- host side ----------------------------------------------------------------

// host formatting of one record with the reference's format strings (the
// records the device left out)
std::string host_record(const Job &J, const std::vector<double> &vals, long r)
{
    char b[512];
    auto co = [](double h, int i) { return h * (i + 0.5); };
    switch (J.layout) {
    case L_PRESSURE: {
        const long nyz = (long)J.ny * J.nz;
        const int i = (int)(r / nyz), j = (int)((r % nyz) / J.nz), k = (int)(r % J.nz);
        std::string s;
        snprintf(b, sizeof(b), "%.6lf %.6lf %.6lf %1.9e\n", co(J.hx, i), co(J.hy, j),
                 co(J.hz, k), vals[0]);
        s = b;
        if (k == J.nz - 1) {
            s += " \n";
            if (j == J.ny - 1) s += " \n";
        }
        return s;
    }
    case L_FLUX: {
        const long nyz = (long)J.ny * J.nz;
        const int i = (int)(r / nyz), j = (int)((r % nyz) / J.nz), k = (int)(r % J.nz);
        snprintf(b, sizeof(b), "%.6lf %.6lf %.6lf %1.9e %1.9e %1.9e \n", co(J.hx, i),
                 co(J.hy, j), co(J.hz, k), vals[0], vals[1], vals[2]);
        return b;
    }
    case L_VTS_VEL:
        snprintf(b, sizeof(b), "%1.8e %1.8e %1.8e\n", vals[0], vals[1], vals[2]);
        return b;
    case L_VTS_PRES:
        snprintf(b, sizeof(b), "%1.8e\n", vals[0]);
        return b;
    case L_VTS_POINTS: {
        const long nxy = (long)J.nx * J.ny;
        const int k = (int)(r / nxy), j = (int)((r % nxy) / J.nx), i = (int)(r % J.nx);
        snprintf(b, sizeof(b), "%.4f %.4f %.4f \n", co(J.hx, i), co(J.hy, j), co(J.hz, k));
        return b;
    }
    case L_KARST_P:
    case L_KARST_U: {
        const int i = (int)r;
        snprintf(b, sizeof(b), "%.6lf %.6lf %.6lf %1.9e\n", co(J.hx, J.x0 + i * J.dx),
                 co(J.hy, J.y0 + i * J.dy), co(J.hz, J.z0 + i * J.dz), vals[0]);
        return b;
    }
    case L_NUM_E:
        snprintf(b, sizeof(b), "%.*e\n", J.prec, vals[0]);
        return b;
    case L_NUM_F:
        snprintf(b, sizeof(b), "%.*f\n", J.prec, vals[0]);
        return b;
    }
    return "";
}

// the values a fallback record prints (read back from the device)
int record_values(const Job &J, long r, std::vector<double> &vals, cudaStream_t st)
{
    vals.clear();
    auto get = [&](const double *p, long i, double *out) {
        return cudaMemcpyAsync(out, p + i, sizeof(double), cudaMemcpyDeviceToHost, st);
    };
    double a = 0, b2 = 0;
    switch (J.layout) {
    case L_PRESSURE: {
        const long nyz = (long)J.ny * J.nz;
        const int i = (int)(r / nyz), j = (int)((r % nyz) / J.nz), k = (int)(r % J.nz);
        HM_CUDA(get(J.p, i + (long)J.nx * (j + (long)J.ny * k), &a));
        break;
    }
    case L_FLUX:
    case L_VTS_VEL: {
        long s = r;
        if (J.layout == L_FLUX) {
            const long nyz = (long)J.ny * J.nz;
            const int i = (int)(r / nyz), j = (int)((r % nyz) / J.nz), k = (int)(r % J.nz);
            s = i + (long)J.nx * (j + (long)J.ny * k);
        }
        hmfem_ele e;
        HM_CUDA(cudaMemcpyAsync(&e, J.v + s, sizeof(e), cudaMemcpyDeviceToHost, st));
        HM_CUDA(cudaStreamSynchronize(st));
        vals = {0.5 * (e.r - e.l), 0.5 * (e.u - e.d), 0.5 * (e.t - e.b)};
        return HMFEM_OK;
    }
    case L_VTS_PRES:
    case L_NUM_E:
    case L_NUM_F:
        HM_CUDA(get(J.p, r, &a));
        break;
    case L_VTS_POINTS:
        return HMFEM_OK;
    case L_KARST_P:
        HM_CUDA(get(J.a, r * J.stride, &a));
        break;
    case L_KARST_U:
        HM_CUDA(get(J.a, r * J.stride, &a));
        HM_CUDA(get(J.b, r * J.stride, &b2));
        HM_CUDA(cudaStreamSynchronize(st));
        vals = {0.5 * (a - b2)};
        return HMFEM_OK;
    }
    HM_CUDA(cudaStreamSynchronize(st));
    vals = {a};
    return HMFEM_OK;
}

// Device buffers and the pinned staging of one writer call.
struct Writer {
    cudaStream_t st = nullptr;
    char *slots = nullptr, *text = nullptr;
    int *len = nullptr, *off = nullptr, *nfall = nullptr, *fall = nullptr;
    char *pin[2] = {nullptr, nullptr};
    cudaEvent_t done[2] = {nullptr, nullptr};
    long pin_used[2] = {0, 0};
    int chunk = 0;

    int open(long maxrec)
    {
        chunk = (int)(maxrec < (1L << 20) ? (maxrec > 0 ? maxrec : 1) : (1L << 20));
        HM_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        HM_CUDA(cudaMalloc(&slots, (size_t)chunk * kSlot));
        HM_CUDA(cudaMalloc(&text, (size_t)chunk * kSlot));
        HM_CUDA(cudaMalloc(&len, sizeof(int) * (chunk + 1)));
        HM_CUDA(cudaMalloc(&off, sizeof(int) * (chunk + 1)));
        HM_CUDA(cudaMalloc(&nfall, sizeof(int)));
        HM_CUDA(cudaMalloc(&fall, sizeof(int) * chunk));
        for (int b = 0; b < 2; b++) {
            HM_CUDA(cudaMallocHost(&pin[b], (size_t)chunk * kSlot));
            HM_CUDA(cudaEventCreateWithFlags(&done[b], cudaEventDisableTiming));
        }
        return HMFEM_OK;
    }

    void close()
    {
        if (st) cudaStreamSynchronize(st);
        cudaFree(slots); cudaFree(text); cudaFree(len); cudaFree(off);
        cudaFree(nfall); cudaFree(fall);
        for (int b = 0; b < 2; b++) {
            if (pin[b]) cudaFreeHost(pin[b]);
            if (done[b]) cudaEventDestroy(done[b]);
        }
        if (st) cudaStreamDestroy(st);
        st = nullptr;
    }

    // formats all records of J; the text goes to f (if non-null) or is
    // appended to out (if non-null)
    int run(const Job &J, FILE *f, std::string *out)
    {
        int slot = 0;
        bool pending[2] = {false, false};
        auto drain = [&](int b) -> int {
            if (!pending[b]) return HMFEM_OK;
            HM_CUDA(cudaEventSynchronize(done[b]));
            if (f && pin_used[b] > 0 &&
                fwrite(pin[b], 1, (size_t)pin_used[b], f) != (size_t)pin_used[b]) {
                set_last_error("file write failed", __FILE__, __LINE__);
                return HMFEM_E_ARG;
            }
            if (out) out->append(pin[b], (size_t)pin_used[b]);
            pending[b] = false;
            return HMFEM_OK;
        };
        for (long r0 = 0; r0 < J.nrec; r0 += chunk) {
            const int m = (int)(J.nrec - r0 < chunk ? J.nrec - r0 : chunk);
            HM_CUDA(cudaMemsetAsync(nfall, 0, sizeof(int), st));
            const int grid = (int)((m + 127) / 128 < 148 * 16 ? (m + 127) / 128 : 148 * 16);
            k_format<<<grid, 128, 0, st>>>(J, r0, m, slots, len, nfall, fall, chunk);
            HM_LAUNCHED();
            int nf = 0;
            HM_CUDA(cudaMemcpyAsync(&nf, nfall, sizeof(int), cudaMemcpyDeviceToHost, st));
            HM_CUDA(cudaStreamSynchronize(st));
            if (nf > 0) {  // rare: NaN / Inf / extreme magnitudes
                std::vector<int> idx(nf);
                HM_CUDA(cudaMemcpyAsync(idx.data(), fall, sizeof(int) * nf,
                                        cudaMemcpyDeviceToHost, st));
                HM_CUDA(cudaStreamSynchronize(st));
                std::vector<double> vals;
                for (int t : idx) {
                    HM_CHECK(record_values(J, r0 + t, vals, st));
                    const std::string s = host_record(J, vals, r0 + t);
                    if ((int)s.size() > kSlot) {
                        set_last_error("line longer than a slot", __FILE__, __LINE__);
                        return HMFEM_E_CAPACITY;
                    }
                    const int l = (int)s.size();
                    HM_CUDA(cudaMemcpyAsync(slots + (long)t * kSlot, s.data(), l,
                                            cudaMemcpyHostToDevice, st));
                    HM_CUDA(cudaMemcpyAsync(len + t, &l, sizeof(int), cudaMemcpyHostToDevice, st));
                    HM_CUDA(cudaStreamSynchronize(st));
                }
            }
            HM_CHECK(scan_exclusive(len, off, m, st));
            k_compact<<<grid, 128, 0, st>>>(m, slots, len, off, text);
            HM_LAUNCHED();
            int last[2];
            HM_CUDA(cudaMemcpyAsync(last, off + m - 1, sizeof(int), cudaMemcpyDeviceToHost, st));
            HM_CUDA(cudaMemcpyAsync(last + 1, len + m - 1, sizeof(int), cudaMemcpyDeviceToHost, st));
            HM_CUDA(cudaStreamSynchronize(st));
            const long total = (long)last[0] + last[1];
            HM_CHECK(drain(slot));  // the buffer this chunk reuses
            HM_CUDA(cudaMemcpyAsync(pin[slot], text, (size_t)total, cudaMemcpyDeviceToHost, st));
            HM_CUDA(cudaEventRecord(done[slot], st));
            pin_used[slot] = total;
            pending[slot] = true;
            slot ^= 1;
        }
        HM_CHECK(drain(slot));
        HM_CHECK(drain(slot ^ 1));
        return HMFEM_OK;
    }
};

// device copy of a host array for the writers (mem 0); `keep` owns it
template <class T>
int device_view(const T *a, long n, int mem, cudaStream_t st, std::vector<void *> &keep,
                const T **out)
{
    if (!a) { *out = nullptr; return HMFEM_OK; }
    if (mem) { *out = a; return HMFEM_OK; }
    void *d = nullptr;
    HM_CUDA(cudaMalloc(&d, sizeof(T) * (n > 0 ? n : 1)));
    keep.push_back(d);
    HM_CUDA(cudaMemcpyAsync(d, a, sizeof(T) * n, cudaMemcpyHostToDevice, st));
    *out = (const T *)d;
    return HMFEM_OK;
}

// One writer call: its buffers, file and the allocation context of this
// thread (the scan draws its temporary storage from it: pointed at the
// writer's stream for the call, restored afterwards).
struct Scope {
    Writer w;
    std::vector<void *> keep;
    FILE *f = nullptr;
    cudaStream_t saved_st = nullptr;
    AllocCache *saved_cache = nullptr;
    bool ctx = false;
    int open(long maxrec)
    {
        HM_CHECK(w.open(maxrec));
        get_alloc_context(&saved_st, &saved_cache);
        set_alloc_context(w.st, nullptr);
        ctx = true;
        return HMFEM_OK;
    }
    ~Scope()
    {
        w.close();
        if (ctx) set_alloc_context(saved_st, saved_cache);
        for (void *p : keep) cudaFree(p);
        if (f) fclose(f);
    }
};

int open_file(Scope &S, const char *path)
{
    S.f = fopen(path, "wb");
    if (!S.f) {
        set_last_error("cannot open the output file", __FILE__, __LINE__);
        return HMFEM_E_ARG;
    }
    return HMFEM_OK;
}

Job grid_job(int layout, int nx, int ny, int nz, double hx, double hy, double hz)
{
    Job J;
    memset(&J, 0, sizeof(J));
    J.layout = layout;
    J.nx = nx; J.ny = ny; J.nz = nz;
    J.hx = hx; J.hy = hy; J.hz = hz;
    J.nrec = (long)nx * ny * nz;
    return J;
}

}  // namespace
}  // namespace hm

extern "C" {

int hmfem_save_pressure(const char *path, int nx, int ny, int nz, double hx, double hy,
                        double hz, const double *p, int mem)
{
    if (!path || !p || nx < 1 || ny < 1 || nz < 1) return HMFEM_E_ARG;
    hm::Scope S;
    hm::Job J = hm::grid_job(hm::L_PRESSURE, nx, ny, nz, hx, hy, hz);
    HM_CHECK(S.open(J.nrec));
    HM_CHECK(hm::device_view(p, J.nrec, mem, S.w.st, S.keep, &J.p));
    HM_CHECK(hm::open_file(S, path));
    return S.w.run(J, S.f, nullptr);
}

int hmfem_save_flux(const char *path, int nx, int ny, int nz, double hx, double hy,
                    double hz, const hmfem_ele *v, int mem)
{
    if (!path || !v || nx < 1 || ny < 1 || nz < 1) return HMFEM_E_ARG;
    hm::Scope S;
    hm::Job J = hm::grid_job(hm::L_FLUX, nx, ny, nz, hx, hy, hz);
    HM_CHECK(S.open(J.nrec));
    HM_CHECK(hm::device_view(v, J.nrec, mem, S.w.st, S.keep, &J.v));
    HM_CHECK(hm::open_file(S, path));
    return S.w.run(J, S.f, nullptr);
}

int hmfem_save_vts(const char *path, int nx, int ny, int nz, double hx, double hy,
                   double hz, const hmfem_ele *v, const double *p, int mem)
{
    if (!path || !v || !p || nx < 1 || ny < 1 || nz < 1) return HMFEM_E_ARG;
    hm::Scope S;
    const long n = (long)nx * ny * nz;
    HM_CHECK(S.open(n));
    hm::Job J = hm::grid_job(hm::L_VTS_VEL, nx, ny, nz, hx, hy, hz);
    HM_CHECK(hm::device_view(v, n, mem, S.w.st, S.keep, &J.v));
    HM_CHECK(hm::device_view(p, n, mem, S.w.st, S.keep, &J.p));
    HM_CHECK(hm::open_file(S, path));
    // vtk.c:22-74, the fixed text around the three blocks
    fprintf(S.f, "<?xml version=\"1.0\"?>\n");
    fprintf(S.f, "<VTKFile type=\"StructuredGrid\" version=\"0.1\">\n");
    fprintf(S.f, "<StructuredGrid WholeExtent=\"0 %d 0 %d 0 %d\">\n", nx - 1, ny - 1, nz - 1);
    fprintf(S.f, "<Piece Extent=\"0 %d 0 %d 0 %d\">\n", nx - 1, ny - 1, nz - 1);
    fprintf(S.f, "<PointData  Vectors=\"Velocity\" Scalars=\"pressure\">\n");
    fprintf(S.f, "<DataArray type=\"Float32\" Name=\"Velocity\" NumberOfComponents=\"3\" "
                 "format=\"ascii\">\n");
    HM_CHECK(S.w.run(J, S.f, nullptr));
    fprintf(S.f, "</DataArray>\n");
    fprintf(S.f, "<DataArray type=\"Float32\" Name=\"pressure\" NumberOfComponents=\"1\" "
                 "format=\"ascii\">\n");
    J.layout = hm::L_VTS_PRES;
    HM_CHECK(S.w.run(J, S.f, nullptr));
    fprintf(S.f, "</DataArray>\n");
    fprintf(S.f, "</PointData>\n");
    fprintf(S.f, "<CellData>\n");
    fprintf(S.f, "</CellData>\n");
    fprintf(S.f, "<Points>\n");
    fprintf(S.f, "<DataArray type=\"Float32\" NumberOfComponents=\"3\">\n");
    J.layout = hm::L_VTS_POINTS;
    HM_CHECK(S.w.run(J, S.f, nullptr));
    fprintf(S.f, "</DataArray>\n");
    fprintf(S.f, "</Points>\n");
    fprintf(S.f, "</Piece>\n");
    fprintf(S.f, "</StructuredGrid>\n");
    fprintf(S.f, "</VTKFile>\n");
    return HMFEM_OK;
}

int hmfem_save_karst(const char *dir, const hmfem_karst *k, double hx, double hy, double hz,
                     const double *pc, const double *ucl, const double *ucr, int mem)
{
    if (!dir || !k || k->number_karst < 0) return HMFEM_E_ARG;
    const int nk = k->number_karst;
    int mmax = 0;
    for (int j = 0; j < nk; j++) {
        if (k->len[j] < 1 || k->pos[j] < 1 || k->pos[j] > 7) {
            hm::set_last_error("conduit length must be >= 1 and position code 1..7",
                               __FILE__, __LINE__);
            return HMFEM_E_ARG;
        }
        if (k->len[j] > mmax) mmax = k->len[j];
    }
    if (nk == 0) return HMFEM_OK;
    hm::Scope S;
    HM_CHECK(S.open(mmax));
    const long mm = (long)mmax * nk;
    const double *dpc = nullptr, *dl = nullptr, *dr = nullptr;
    HM_CHECK(hm::device_view(pc, mm, mem, S.w.st, S.keep, &dpc));
    HM_CHECK(hm::device_view(ucl, mm, mem, S.w.st, S.keep, &dl));
    HM_CHECK(hm::device_view(ucr, mm, mem, S.w.st, S.keep, &dr));
    // posprocessing_output.c:451-520: direction of each position code
    static const int DX[8] = {0, 1, 0, 0, 1, 1, -1, -1};
    static const int DY[8] = {0, 0, 1, 0, 1, -1, 1, -1};
    static const int DZ[8] = {0, 0, 0, 1, 0, 0, 0, 0};
    for (int kind = 0; kind < 2; kind++) {
        const double *a = kind == 0 ? dpc : dr, *b = kind == 0 ? nullptr : dl;
        if (!a || (kind == 1 && !b)) continue;
        for (int j = 0; j < nk; j++) {
            char path[4096];
            snprintf(path, sizeof(path), "%s/%s_karst_%i.dat", dir,
                     kind == 0 ? "pressure" : "flux", j);
            FILE *f = fopen(path, "wb");
            if (!f) {
                hm::set_last_error("cannot open a conduit output file", __FILE__, __LINE__);
                return HMFEM_E_ARG;
            }
            hm::Job J;
            memset(&J, 0, sizeof(J));
            J.layout = kind == 0 ? hm::L_KARST_P : hm::L_KARST_U;
            J.nrec = k->len[j];
            J.hx = hx; J.hy = hy; J.hz = hz;
            J.x0 = k->sxi[j]; J.y0 = k->syi[j]; J.z0 = k->szi[j];
            J.dx = DX[k->pos[j]]; J.dy = DY[k->pos[j]]; J.dz = DZ[k->pos[j]];
            J.a = a + j;
            J.b = b ? b + j : nullptr;
            J.stride = nk;
            const int rc = S.w.run(J, f, nullptr);
            fclose(f);
            if (rc != HMFEM_OK) return rc;
        }
    }
    return HMFEM_OK;
}

int hmfem_format_numbers(const double *x, long n, char conv, int prec, char *out, long cap,
                         long *used, int mem)
{
    if (!x || n < 0 || !out || cap < 0 || prec < 0 || prec > 17 ||
        (conv != 'e' && conv != 'f'))
        return HMFEM_E_ARG;
    hm::Scope S;
    hm::Job J;
    memset(&J, 0, sizeof(J));
    J.layout = conv == 'e' ? hm::L_NUM_E : hm::L_NUM_F;
    J.nrec = n;
    J.prec = prec;
    HM_CHECK(S.open(n));
    HM_CHECK(hm::device_view(x, n, mem, S.w.st, S.keep, &J.p));
    std::string text;
    if (n > 0) HM_CHECK(S.w.run(J, nullptr, &text));
    if (used) *used = (long)text.size();
    if ((long)text.size() > cap) {
        hm::set_last_error("output buffer too small", __FILE__, __LINE__);
        return HMFEM_E_CAPACITY;
    }
    memcpy(out, text.data(), text.size());
    return HMFEM_OK;
}

}  // extern "C"
