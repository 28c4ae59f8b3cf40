// k_text.cu — the *.prof and *.vtk writers on the device.
//
// The reference prints every particle with fprintf "%e" / "%d" on the host
// (writeProfFile, main.cpp:672-696; writeVtkFile, main.cpp:698-834).  Here a
// document is a list of sections, each a header string followed by one
// record per particle; three launches turn it into the file's bytes in device
// memory: (1) every record's length (from the value's sign and magnitude, no
// digits), summed per block; (2) one block scans the block sums into byte
// offsets; (3) every record is formatted into shared memory at its offset and
// the block's text is stored with aligned 16-byte stores.  The host then copies the bytes out and writes them
// with one fwrite.
//
// "%e" is exact: the digits equal glibc's (the decimal value of the double,
// rounded to 7 significant digits, ties to even).  The fast path multiplies by
// 10^s held as a double-double (relative error < 2^-104); it decides the
// rounding unless the scaled value lies within 2^-70 of a half-integer, and
// there an exact big-integer comparison decides.
#include <cuda_runtime.h>
#include <stdint.h>

#include "mph_pow10.h"
#include "mph_text.h"

namespace mph {
namespace {

constexpr int kTextThreads = kTextBlockUnits;  // threads per block, one unit each
// A block's text: at most one header and 255 records, or 256 records, plus
// the 15-byte alignment lead and one unit of slack.
constexpr int kTextStageBytes = (kTextMaxUnit + 255 * 103 + 15 + kTextMaxUnit + 15) / 16 * 16;
static_assert(kTextMaxRecord[kRecProf] == 103, "stage bound assumes the longest record is 103 bytes");
constexpr int kBigWords = 32;      // 1024-bit integers: the exact path needs < 860 bits

// ---- exact comparison (slow path) ------------------------------------------
struct Big {
    uint32_t w[kBigWords];
    int len;
};

__device__ void big_set(Big& b, uint64_t v) {
    b.w[0] = (uint32_t)v;
    b.w[1] = (uint32_t)(v >> 32);
    b.len = b.w[1] ? 2 : (b.w[0] ? 1 : 0);
}

__device__ void big_mul(Big& b, uint32_t k) {
    uint64_t carry = 0;
    for (int i = 0; i < b.len; ++i) {
        const uint64_t t = (uint64_t)b.w[i] * k + carry;
        b.w[i] = (uint32_t)t;
        carry = t >> 32;
    }
    if (carry && b.len < kBigWords) b.w[b.len++] = (uint32_t)carry;
}

__device__ void big_mul_pow5(Big& b, int k) {
    for (; k >= 13; k -= 13) big_mul(b, 1220703125u);  // 5^13
    uint32_t p = 1;
    for (; k > 0; --k) p *= 5;
    big_mul(b, p);
}

__device__ void big_shl(Big& b, int sh) {
    if (b.len == 0 || sh <= 0) return;
    const int ws = sh >> 5, bs = sh & 31;
    int top = b.len + ws + 1;
    if (top > kBigWords) top = kBigWords;
    for (int i = top - 1; i >= 0; --i) {
        const int src = i - ws;
        uint32_t v = 0;
        if (src >= 0 && src < b.len) v = b.w[src] << bs;
        if (bs && src - 1 >= 0 && src - 1 < b.len) v |= b.w[src - 1] >> (32 - bs);
        b.w[i] = v;
    }
    b.len = top;
    while (b.len > 0 && b.w[b.len - 1] == 0) --b.len;
}

__device__ int big_cmp(const Big& a, const Big& b) {
    if (a.len != b.len) return a.len < b.len ? -1 : 1;
    for (int i = a.len - 1; i >= 0; --i)
        if (a.w[i] != b.w[i]) return a.w[i] < b.w[i] ? -1 : 1;
    return 0;
}

// sign of m * 2^e * 10^s - (n + 1/2), exactly.
__device__ __noinline__ int cmp_half_exact(uint64_t m, int e, int s, uint32_t n) {
    Big l, r;
    big_set(l, m);
    big_mul(l, 2);
    big_set(r, 2ull * n + 1);
    int p2 = e + s;  // 2m*2^e*10^s = 2m*5^s*2^(e+s)
    if (s >= 0)
        big_mul_pow5(l, s);
    else
        big_mul_pow5(r, -s);
    if (p2 >= 0)
        big_shl(l, p2);
    else
        big_shl(r, -p2);
    return big_cmp(l, r);
}

// ---- "%e" and "%d" -----------------------------------------------------------
__device__ __forceinline__ int put_digits(char* o, uint32_t v) {  // v > 0 or a lone 0
    char t[10];
    int k = 0;
    do {
        t[k++] = (char)('0' + v % 10);
        v /= 10;
    } while (v);
    for (int i = 0; i < k; ++i) o[i] = t[k - 1 - i];
    return k;
}

__device__ __forceinline__ int fmt_int(char* o, int v) {
    int k = 0;
    uint32_t u = (uint32_t)v;
    if (v < 0) {
        o[k++] = '-';
        u = 0u - u;
    }
    return k + put_digits(o + k, u);
}

__device__ __forceinline__ int put_mantissa_exp(char* o, uint32_t r, int E) {
    // r in [10^6, 10^7): d.dddddd e(+|-)XX[X]
    char d[7];
    for (int i = 6; i >= 0; --i) {
        d[i] = (char)('0' + r % 10);
        r /= 10;
    }
    o[0] = d[0];
    o[1] = '.';
    for (int i = 1; i < 7; ++i) o[1 + i] = d[i];
    o[8] = 'e';
    o[9] = E < 0 ? '-' : '+';
    uint32_t a = (uint32_t)(E < 0 ? -E : E);
    int k = 10;
    if (a >= 100) {
        o[k++] = (char)('0' + a / 100);
        a %= 100;
    }
    o[k++] = (char)('0' + a / 10);
    o[k++] = (char)('0' + a % 10);
    return k;
}

// x * 10^s as hi + lo (|error| < 2^-104 * x * 10^s).
__device__ __forceinline__ void scaled(double x, int s, double& qh, double& ql) {
    const double2 t = kMphPow10[s - MPH_POW10_MIN];
    const double xs = s > 250 ? x * 0x1p256 : (s < -250 ? x * 0x1p-256 : x);
    const double p = xs * t.x;
    const double pe = fma(xs, t.x, -p);
    const double c = fma(xs, t.y, pe);
    qh = p + c;
    ql = c - (qh - p);
}

// printf("%e", x) into o; returns the length (at most 14).
__device__ int fmt_e(char* o, double x) {
    const uint64_t bits = (uint64_t)__double_as_longlong(x);
    int k = 0;
    if (bits >> 63) o[k++] = '-';
    const int be = (int)((bits >> 52) & 0x7ff);
    const uint64_t fr = bits & ((1ull << 52) - 1);
    if (be == 0x7ff) {
        o[k] = fr ? 'n' : 'i';
        o[k + 1] = fr ? 'a' : 'n';
        o[k + 2] = fr ? 'n' : 'f';
        return k + 3;
    }
    if (be == 0 && fr == 0) return k + put_mantissa_exp(o + k, 0, 0);
    const uint64_t m = be ? (fr | (1ull << 52)) : fr;
    const int e = be ? be - 1075 : -1074;  // |x| = m * 2^e
    const double ax = fabs(x);
    const int e2 = e + 63 - __clzll((long long)m);  // floor(log2 |x|)
    int E = (e2 * 78913) >> 18;                     // ~floor(e2 * log10(2)), corrected below
    double qh, ql;
    scaled(ax, 6 - E, qh, ql);
    if (qh < 1.0e6) {
        --E;
        scaled(ax, 6 - E, qh, ql);
    } else if (qh >= 1.0e7) {
        ++E;
        scaled(ax, 6 - E, qh, ql);
    }
    const double fl = floor(qh);
    uint32_t r = (uint32_t)fl;
    const double f = qh - fl;  // exact
    bool up;
    if (f != 0.5) {
        up = f > 0.5;
    } else if (fabs(ql) > 0x1p-70) {
        up = ql > 0.0;
    } else {
        const int c = cmp_half_exact(m, e, 6 - E, r);
        up = c > 0 || (c == 0 && (r & 1u));
    }
    r += up ? 1u : 0u;
    if (r >= 10000000u) {
        r = 1000000u;
        ++E;
    }
    return k + put_mantissa_exp(o + k, r, E);
}

__device__ __forceinline__ int fmt_e_float(char* o, double x) { return fmt_e(o, (double)__double2float_rn(x)); }

// Lengths without the digits: "%e" is 12 characters plus the sign while the
// printed exponent has two digits, which holds for every value in
// [1.0000001e-99, 9.9e99) and for every float; outside that range the value
// is formatted to be measured.
__device__ __forceinline__ int len_e(double x) {
    const uint64_t bits = (uint64_t)__double_as_longlong(x);
    const int sign = (int)(bits >> 63);
    if (((bits >> 52) & 0x7ff) == 0x7ff) return sign + 3;
    const double ax = fabs(x);
    if (ax == 0.0 || (ax >= 1.0000001e-99 && ax < 9.9e99)) return sign + 12;
    char t[16];
    return fmt_e(t, x);
}

__device__ __forceinline__ int len_e_float(double x) { return len_e((double)__double2float_rn(x)); }

__device__ __forceinline__ int len_uint(uint32_t v) {
    int k = 1;
    while (v >= 10) {
        v /= 10;
        ++k;
    }
    return k;
}

__device__ __forceinline__ int len_int(int v) { return v < 0 ? 1 + len_uint(0u - (uint32_t)v) : len_uint((uint32_t)v); }

// ---- records -------------------------------------------------------------------
// One record of a section: the particle's line in the reference's format.
__device__ int format_record(const TextSection& s, int i, char* o) {
    int k = 0;
    switch (s.kind) {
        case kRecProf: {  // "%d %e %e %e  %e %e %e\n" (writeProfFile)
            const double4 q = reinterpret_cast<const double4*>(s.src0)[i];
            const double4 v = reinterpret_cast<const double4*>(s.src1)[i];
            k += fmt_int(o + k, reinterpret_cast<const int*>(s.src2)[i]);
            o[k++] = ' ';
            k += fmt_e(o + k, q.x);
            o[k++] = ' ';
            k += fmt_e(o + k, q.y);
            o[k++] = ' ';
            k += fmt_e(o + k, q.z);
            o[k++] = ' ';
            o[k++] = ' ';
            k += fmt_e(o + k, v.x);
            o[k++] = ' ';
            k += fmt_e(o + k, v.y);
            o[k++] = ' ';
            k += fmt_e(o + k, v.z);
            o[k++] = '\n';
            break;
        }
        case kRecVec3f: {  // "%e %e %e\n" of (float) components
            const double4 q = reinterpret_cast<const double4*>(s.src0)[i];
            k += fmt_e_float(o + k, q.x);
            o[k++] = ' ';
            k += fmt_e_float(o + k, q.y);
            o[k++] = ' ';
            k += fmt_e_float(o + k, q.z);
            o[k++] = '\n';
            break;
        }
        case kRecScalarf:  // "%e\n" of (float)
            k += fmt_e_float(o + k, reinterpret_cast<const double*>(s.src0)[i]);
            o[k++] = '\n';
            break;
        case kRecScalard:  // "%e\n"
            k += fmt_e(o + k, reinterpret_cast<const double*>(s.src0)[i]);
            o[k++] = '\n';
            break;
        case kRecInt:  // "%d\n"
            k += fmt_int(o + k, reinterpret_cast<const int*>(s.src0)[i]);
            o[k++] = '\n';
            break;
        case kRecCell:  // "1 %d "
            o[k++] = '1';
            o[k++] = ' ';
            k += fmt_int(o + k, i);
            o[k++] = ' ';
            break;
        case kRecOne:  // "1 "
            o[k++] = '1';
            o[k++] = ' ';
            break;
        default:
            break;
    }
    return k;
}

// The length format_record gives, computed without formatting.
__device__ int record_len(const TextSection& s, int i) {
    switch (s.kind) {
        case kRecProf: {
            const double4 q = reinterpret_cast<const double4*>(s.src0)[i];
            const double4 v = reinterpret_cast<const double4*>(s.src1)[i];
            return len_int(reinterpret_cast<const int*>(s.src2)[i]) + len_e(q.x) + len_e(q.y) + len_e(q.z) +
                   len_e(v.x) + len_e(v.y) + len_e(v.z) + 8;
        }
        case kRecVec3f: {
            const double4 q = reinterpret_cast<const double4*>(s.src0)[i];
            return len_e_float(q.x) + len_e_float(q.y) + len_e_float(q.z) + 3;
        }
        case kRecScalarf:
            return len_e_float(reinterpret_cast<const double*>(s.src0)[i]) + 1;
        case kRecScalard:
            return len_e(reinterpret_cast<const double*>(s.src0)[i]) + 1;
        case kRecInt:
            return len_int(reinterpret_cast<const int*>(s.src0)[i]) + 1;
        case kRecCell:
            return len_int(i) + 3;
        case kRecOne:
            return 2;
        default:
            return 0;
    }
}

// Unit u of section s: 0 is the header, u >= 1 the record of particle u - 1.
__device__ __forceinline__ int format_unit(const TextDoc& d, const TextSection& s, int u, char* o) {
    if (u == 0) {
        for (int c = 0; c < s.head_len; ++c) o[c] = d.head[s.head_off + c];
        return s.head_len;
    }
    return format_record(s, u - 1, o);
}

__device__ __forceinline__ int find_section(const TextDoc& d, int b) {
    int k = 0;
    while (k + 1 < d.nsec && d.sec[k + 1].first_block <= b) ++k;
    return k;
}

// Pass 1: every unit's length (kept for pass 3) and the block's sum.
__global__ void __launch_bounds__(kTextThreads) k_text_count(const __grid_constant__ TextDoc d,
                                                             uint16_t* __restrict__ unit_len,
                                                             uint32_t* __restrict__ blk_bytes) {
    const int b = blockIdx.x;
    const TextSection& s = d.sec[find_section(d, b)];
    const int u = (b - s.first_block) * kTextThreads + threadIdx.x;
    uint32_t len = 0;
    if (u == 0)
        len = (uint32_t)s.head_len;
    else if (u <= s.n)
        len = (uint32_t)record_len(s, u - 1);
    unit_len[(size_t)b * kTextThreads + threadIdx.x] = (uint16_t)len;
    for (int o = 16; o > 0; o >>= 1) len += __shfl_xor_sync(0xffffffffu, len, o);
    __shared__ uint32_t ws[kTextThreads / 32];
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = len;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t t = 0;
        for (int w = 0; w < kTextThreads / 32; ++w) t += ws[w];
        blk_bytes[b] = t;
    }
}

// One block: exclusive scan of the block byte counts; total in off[nblocks].
// Each thread takes 16 consecutive counts (four 16-byte loads) per pass.
__global__ void __launch_bounds__(1024) k_text_scan(const uint32_t* __restrict__ blk_bytes,
                                                    unsigned long long* __restrict__ off, int nblocks) {
    constexpr int kPer = 16;
    __shared__ unsigned long long ws[32];
    __shared__ unsigned long long carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int base = 0; base < nblocks; base += 1024 * kPer) {
        const int i0 = base + threadIdx.x * kPer;
        uint32_t v[kPer];
        if (i0 + kPer <= nblocks) {
            const uint4* p = reinterpret_cast<const uint4*>(blk_bytes + i0);  // i0 is a multiple of 16
#pragma unroll
            for (int q = 0; q < kPer / 4; ++q) {
                const uint4 t = p[q];
                v[4 * q] = t.x;
                v[4 * q + 1] = t.y;
                v[4 * q + 2] = t.z;
                v[4 * q + 3] = t.w;
            }
        } else {
#pragma unroll
            for (int q = 0; q < kPer; ++q) v[q] = i0 + q < nblocks ? blk_bytes[i0 + q] : 0u;
        }
        unsigned long long sum = 0;
#pragma unroll
        for (int q = 0; q < kPer; ++q) sum += v[q];
        unsigned long long x = sum;
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned long long y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) ws[w] = x;
        __syncthreads();
        if (w == 0) {
            unsigned long long t = ws[lane];
            for (int o = 1; o < 32; o <<= 1) {
                const unsigned long long y = __shfl_up_sync(0xffffffffu, t, o);
                if (lane >= o) t += y;
            }
            ws[lane] = t;  // inclusive over warps
        }
        __syncthreads();
        const unsigned long long incl = x + (w ? ws[w - 1] : 0ull) + carry;
        unsigned long long run = incl - sum;
#pragma unroll
        for (int q = 0; q < kPer; ++q) {
            if (i0 + q < nblocks) off[i0 + q] = run;
            run += v[q];
        }
        __syncthreads();
        if (threadIdx.x == 1023) carry = incl;
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        off[nblocks] = carry;
        off[nblocks + 1] = 0;  // the length-mismatch flag of pass 3
    }
}

// Pass 3: every unit formatted into shared memory at its offset within the
// block, then the block's bytes stored with aligned 16-byte stores (bytes at
// the two ragged ends).  A unit whose text differs in length from pass 1 sets
// off[nblocks + 1].
__global__ void __launch_bounds__(kTextThreads) k_text_write(const __grid_constant__ TextDoc d,
                                                             const uint16_t* __restrict__ unit_len,
                                                             unsigned long long* __restrict__ off,
                                                             char* __restrict__ out) {
    __shared__ __align__(16) char stage[kTextStageBytes];
    __shared__ uint32_t ws[kTextThreads / 32];
    const int b = blockIdx.x;
    const TextSection& s = d.sec[find_section(d, b)];
    const int u = (b - s.first_block) * kTextThreads + threadIdx.x;
    const uint32_t len = unit_len[(size_t)b * kTextThreads + threadIdx.x];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    uint32_t x = len;
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) ws[w] = x;
    __syncthreads();
    uint32_t before = 0, total = 0;
    for (int k = 0; k < kTextThreads / 32; ++k) {
        before += k < w ? ws[k] : 0u;
        total += ws[k];
    }
    const unsigned long long base = off[b];
    const int a = (int)(base & 15ull);
    if (u <= s.n) {
        const int got = format_unit(d, s, u, stage + a + before + (x - len));
        if (got != (int)len) atomicOr(reinterpret_cast<unsigned int*>(off + d.nblocks + 1), 1u);
    }
    __syncthreads();
    char* g = out + (base - (unsigned long long)a);  // 16-byte aligned
    const int end = a + (int)total;
    for (int lo = threadIdx.x * 16; lo < end; lo += kTextThreads * 16) {
        if (lo >= a && lo + 16 <= end) {
            *reinterpret_cast<uint4*>(g + lo) = *reinterpret_cast<const uint4*>(stage + lo);
        } else {
            const int c1 = lo + 16 < end ? lo + 16 : end;
            for (int c = lo > a ? lo : a; c < c1; ++c) g[c] = stage[c];
        }
    }
}

// Values as "%e\n" lines (as_float: each cast to float first, as writeVtkFile
// prints), for testing the formatter against the host's printf.
__global__ void __launch_bounds__(kTextThreads) k_text_values(const double* __restrict__ v, long long n, int as_float,
                                                              char* __restrict__ out) {
    const long long i = (long long)blockIdx.x * kTextThreads + threadIdx.x;
    if (i >= n) return;
    char* o = out + i * kTextValueStride;
    const int k = as_float ? fmt_e_float(o + 1, v[i]) : fmt_e(o + 1, v[i]);
    o[1 + k] = '\n';
    o[0] = (char)(k + 1);
}

}  // namespace

int text_blocks(TextDoc& d) {
    int b = 0;
    for (int k = 0; k < d.nsec; ++k) {
        d.sec[k].first_block = b;
        b += (d.sec[k].n + 1 + kTextThreads - 1) / kTextThreads;  // header + records
    }
    d.nblocks = b;
    return b;
}

size_t text_max_bytes(const TextDoc& d) {
    size_t t = 0;
    for (int k = 0; k < d.nsec; ++k) t += (size_t)d.sec[k].head_len + (size_t)d.sec[k].n * kTextMaxRecord[d.sec[k].kind];
    return t;
}

int launch_text(const TextDoc& d, uint16_t* unit_len, uint32_t* blk_bytes, unsigned long long* off, char* out,
                cudaStream_t s) {
    if (d.nblocks <= 0) return 0;
    k_text_count<<<d.nblocks, kTextThreads, 0, s>>>(d, unit_len, blk_bytes);
    k_text_scan<<<1, 1024, 0, s>>>(blk_bytes, off, d.nblocks);
    k_text_write<<<d.nblocks, kTextThreads, 0, s>>>(d, unit_len, off, out);
    return 3;
}

void launch_text_values(const double* v, long long n, int as_float, char* out, cudaStream_t s) {
    if (n <= 0) return;
    k_text_values<<<(unsigned)((n + kTextThreads - 1) / kTextThreads), kTextThreads, 0, s>>>(v, n, as_float, out);
}

}  // namespace mph
