// ingest.cu -- sparse tensor files parsed on the GPU.
//
// The reference reads a tensor on the host (src/sptensor/load.c:63-265):
// text coordinate files with fscanf, one "%u" per index and one "%lf" per
// value, and SPLATT binary files with fread.  Here the file's bytes are copied
// to the device in pinned chunks and parsed there:
//
//   text:   tok_count_kernel   token starts per 16 KB chunk (a token is a run
//                              of bytes other than the six C-locale spaces)
//           scan               first token ordinal of every chunk
//           tok_parse_kernel   every token parsed where it starts; token t
//                              after the header is field t % (N+1) of nonzero
//                              t / (N+1) and goes straight to its array
//   binary: header on the host; index and value sections copied on the device
//           (FP64 values rounded to FP32 by a kernel)
//
// Results are those of the reference's loader:
//   - an index token is read as fscanf("%u") reads it: optional sign, decimal
//     digits, the value taken modulo 2^32 (a negative number wraps; one that
//     overflows 64 bits becomes 0xFFFFFFFF); start_index is subtracted, and an
//     index below start_index is an error;
//   - a value token is read as glibc's fscanf("%lf") reads it: the decimal
//     number is rounded correctly to FP64 (Clinger's exact fast path when the
//     digits fit 2^53 and the power of ten is exact, otherwise an exact
//     big-integer quotient), then to FP32; "inf", "infinity" and "nan" are
//     accepted, and an exponent marker without digits ("1e", "2.5e+") is
//     consumed and leaves the mantissa's value;
//   - reading stops at the first token that is not entirely a number, as
//     fscanf does: the nonzero holding it is dropped, unless it is a value
//     whose leading part is a number (then fscanf has read that nonzero and
//     fails on the next one).  A trailing incomplete nonzero is dropped.
// Deliberate limits (reported as errors instead of being parsed): hexadecimal
// values, "nan(...)" payloads, values with more than 100 significant digits
// and tokens longer than 4096 bytes.  Two numbers written without white space
// between them ("12-5") are one malformed token here; fscanf would read two.
//
// Duplicate coordinates are kept, as the reference keeps them.  On request
// (ptiB200LoadSparseTensor's dedupe) the nonzeros are sorted by coordinate
// (mode 0 most significant, ties in file order) and each run of one
// coordinate becomes one nonzero whose value is the FP32 sum of the run's
// values in file order.
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <fcntl.h>
#include <mutex>
#include <sys/stat.h>
#include <thread>
#include <unistd.h>

#include "primitives.cuh"
#include "tensor.cuh"

namespace pti {

namespace {

constexpr int kIngThreads = 256;
constexpr int kIngSeg = 16;                                     // bytes per thread per step
constexpr int kIngSteps = 4;                                    // steps per chunk
constexpr int kIngStep = kIngThreads * kIngSeg;                 // 4 KB
constexpr int kIngChunk = kIngStep * kIngSteps;                 // 16 KB per CTA
constexpr uint32_t kMaxToken = 4096;
constexpr int kMaxSigDigits = 100;
constexpr size_t kReadChunk = 16ull << 20;                      // pinned read buffer

// Error flags of the parse (bit set in ParseSlots::fatal_flags)
constexpr uint32_t kFatalHex = 1, kFatalNanPayload = 2, kFatalLong = 4, kFatalDigits = 8;

struct ParseSlots {
    unsigned long long bad;    // min over malformed tokens of ordinal*2 + (value with a number prefix)
    unsigned long long low;    // min ordinal of an index read below start_index
    unsigned long long fatal;  // min ordinal of a token the parser refuses
    unsigned int fatal_flags;
    unsigned int pad;
};

__device__ __forceinline__ bool is_ws(uint32_t c) { return c == ' ' || (c >= 9 && c <= 13); }
__device__ __forceinline__ bool is_digit(uint32_t c) { return c - '0' < 10u; }
__device__ __forceinline__ uint32_t lower(uint32_t c) { return c | 0x20u; }

// Bit i set: byte off+i starts a token.  The buffer is padded with spaces to a
// whole number of chunks (+64 bytes).
__device__ __forceinline__ uint32_t seg_starts(const uint8_t *buf, uint64_t off)
{
    const uint4 v = *reinterpret_cast<const uint4 *>(buf + off);
    const uint32_t w[4] = {v.x, v.y, v.z, v.w};
    uint32_t nonws = 0;
#pragma unroll
    for (int i = 0; i < 16; ++i) nonws |= (is_ws((w[i >> 2] >> ((i & 3) * 8)) & 0xFFu) ? 0u : 1u) << i;
    const uint32_t prev = off ? (is_ws(buf[off - 1]) ? 0u : 1u) : 0u;
    return nonws & ~((nonws << 1) | prev);
}

__global__ void __launch_bounds__(kIngThreads) tok_count_kernel(const uint8_t *buf, uint32_t *counts)
{
    __shared__ uint32_t s_warp[kIngThreads / 32];
    const uint64_t base = (uint64_t)blockIdx.x * kIngChunk;
    uint32_t c = 0;
#pragma unroll
    for (int j = 0; j < kIngSteps; ++j) c += __popc(seg_starts(buf, base + (uint64_t)j * kIngStep + threadIdx.x * kIngSeg));
    uint32_t total;
    block_exclusive_scan<uint32_t>(c, s_warp, total);
    if (threadIdx.x == 0) counts[blockIdx.x] = total;
}

struct CountIn {
    const uint32_t *c;
    __device__ uint64_t operator()(uint64_t i) const { return c[i]; }
};
struct OffsetOut {
    uint64_t *o;
    __device__ void operator()(uint64_t i, uint64_t prefix, uint64_t) const { o[i] = prefix; }
};

// ---------------------------------------------------------------------------
// Token parsers
// ---------------------------------------------------------------------------
struct IndexTok {
    uint32_t value;
    bool prefix_ok;  // at least one digit was read
    bool whole;      // the number is the whole token
};

__device__ IndexTok parse_index(const uint8_t *p, uint32_t len)
{
    uint32_t i = 0;
    bool neg = false;
    if (i < len && (p[i] == '+' || p[i] == '-')) neg = p[i++] == '-';
    uint64_t v = 0;
    bool over = false;
    const uint32_t d0 = i;
    for (; i < len && is_digit(p[i]); ++i) {
        const uint64_t d = p[i] - '0';
        if (v > (~0ull - d) / 10) over = true;
        else v = v * 10 + d;
    }
    IndexTok r;
    r.prefix_ok = i > d0;
    r.whole = r.prefix_ok && i == len;
    // strtoul: out of range -> ULONG_MAX (sign ignored); else the negation
    // modulo 2^64.  fscanf then stores the low 32 bits.
    r.value = over ? 0xFFFFFFFFu : (uint32_t)(neg ? (0ull - v) : v);
    return r;
}

// Multi-limb unsigned integers for the exact conversion (little-endian u32).
constexpr int kLimbs = 24;  // 768 bits: up to 100 digits times 2^(-e) or 10^147 times 2^55
struct Big {
    uint32_t l[kLimbs];
    int n;  // limbs in use
};

__device__ void big_set(Big &a, uint64_t v)
{
    a.l[0] = (uint32_t)v;
    a.l[1] = (uint32_t)(v >> 32);
    a.n = a.l[1] ? 2 : (a.l[0] ? 1 : 0);
}
__device__ void big_mul_small(Big &a, uint32_t m, uint32_t add)
{
    uint64_t carry = add;
    for (int i = 0; i < a.n; ++i) {
        const uint64_t t = (uint64_t)a.l[i] * m + carry;
        a.l[i] = (uint32_t)t;
        carry = t >> 32;
    }
    if (carry && a.n < kLimbs) a.l[a.n++] = (uint32_t)carry;
}
__device__ int big_bits(const Big &a)
{
    return a.n ? (a.n - 1) * 32 + (32 - __clz(a.l[a.n - 1])) : 0;
}
__device__ void big_shl(Big &a, int s)
{
    if (!a.n || s <= 0) return;
    const int w = s >> 5, b = s & 31;
    int n = a.n + w + 1;
    if (n > kLimbs) n = kLimbs;
    for (int i = n - 1; i >= 0; --i) {
        const int j = i - w;
        uint32_t hi = (j >= 0 && j < a.n) ? a.l[j] : 0u;
        uint32_t lo = (j - 1 >= 0 && j - 1 < a.n) ? a.l[j - 1] : 0u;
        a.l[i] = b ? (hi << b) | (lo >> (32 - b)) : hi;
    }
    a.n = n;
    while (a.n && !a.l[a.n - 1]) --a.n;
}
__device__ void big_shr1(Big &a)
{
    for (int i = 0; i < a.n; ++i) a.l[i] = (a.l[i] >> 1) | (i + 1 < a.n ? a.l[i + 1] << 31 : 0u);
    while (a.n && !a.l[a.n - 1]) --a.n;
}
__device__ int big_cmp(const Big &a, const Big &b)
{
    if (a.n != b.n) return a.n < b.n ? -1 : 1;
    for (int i = a.n - 1; i >= 0; --i)
        if (a.l[i] != b.l[i]) return a.l[i] < b.l[i] ? -1 : 1;
    return 0;
}
__device__ void big_sub(Big &a, const Big &b)  // a -= b, a >= b
{
    int64_t borrow = 0;
    for (int i = 0; i < a.n; ++i) {
        int64_t t = (int64_t)a.l[i] - (i < b.n ? (int64_t)b.l[i] : 0) - borrow;
        borrow = t < 0;
        a.l[i] = (uint32_t)(t + (borrow << 32));
    }
    while (a.n && !a.l[a.n - 1]) --a.n;
}

// The FP64 nearest to D * 10^q, D > 0 being the nd significant digits of the
// mantissa at p (leading zeros and the decimal point are skipped), for values
// whose FP32 rounding is not simply 0 or infinity: 10^-48 <= value < 10^39.
// Exact: num / den with num, den integers, quotient bits by restoring
// division, round half to even with the remainder as sticky bit.
__device__ double exact_decimal(const uint8_t *p, int nd, int q)
{
    Big num, den;
    big_set(num, 0);
    for (int got = 0; got < nd; ++p) {
        const uint32_t c = *p;
        if (!is_digit(c) || (got == 0 && c == '0')) continue;  // '.', leading zeros
        big_mul_small(num, 10, c - '0');
        ++got;
    }
    big_set(den, 1);
    if (q >= 0)
        for (int i = 0; i < q; ++i) big_mul_small(num, 10, 0);
    else
        for (int i = 0; i < -q; ++i) big_mul_small(den, 10, 0);
    // scale so that the quotient has 54 or 55 bits
    int e = big_bits(num) - big_bits(den) - 54;
    if (e < 0) big_shl(num, -e);
    else big_shl(den, e);
    Big dd = den;
    big_shl(dd, 54);
    uint64_t Q = 0;
    for (int bit = 54; bit >= 0; --bit) {
        if (big_cmp(num, dd) >= 0) {
            big_sub(num, dd);
            Q |= 1ull << bit;
        }
        big_shr1(dd);
    }
    bool sticky = num.n != 0;
    while (Q >= (1ull << 54)) {
        sticky |= Q & 1;
        Q >>= 1;
        ++e;
    }
    // Q in [2^53, 2^54): 53 bits and a round bit; value = Q * 2^e
    uint64_t m = Q >> 1;
    if ((Q & 1) && (sticky || (m & 1))) ++m;
    int ex = e + 1;
    if (m == (1ull << 53)) {
        m >>= 1;
        ++ex;
    }
    // m in [2^52, 2^53): value = m * 2^ex, a normal double in this range
    const uint64_t bits = ((uint64_t)(ex + 52 + 1023) << 52) | (m & ((1ull << 52) - 1));
    return __longlong_as_double((long long)bits);
}

struct ValueTok {
    float value;
    bool prefix_ok;  // fscanf's "%lf" reads a number from the token's start
    bool whole;
    uint32_t fatal;  // kFatal* bits
};

__device__ ValueTok parse_value(const uint8_t *p, uint32_t len)
{
    ValueTok r{0.f, false, false, 0u};
    uint32_t i = 0;
    bool neg = false;
    if (i < len && (p[i] == '+' || p[i] == '-')) neg = p[i++] == '-';
    // inf / infinity / nan (case-insensitive)
    if (i < len && (lower(p[i]) == 'i' || lower(p[i]) == 'n')) {
        auto match = [&](const char *w, uint32_t at) {
            uint32_t k = 0;
            for (; w[k]; ++k)
                if (at + k >= len || lower(p[at + k]) != (uint32_t)w[k]) return 0u;
            return k;
        };
        uint32_t k = match("infinity", i);
        // "inf" followed by an 'i' that does not complete "infinity" is no number
        if (!k && (k = match("inf", i)) && i + k < len && lower(p[i + k]) == 'i') return r;
        if (k) {
            r.value = neg ? -__int_as_float(0x7f800000) : __int_as_float(0x7f800000);
            r.prefix_ok = true;
            r.whole = i + k == len;
            return r;
        }
        if ((k = match("nan", i))) {
            if (i + k < len && p[i + k] == '(') {
                r.fatal = kFatalNanPayload;
                return r;
            }
            r.value = __int_as_float(neg ? (int)0xffc00000 : 0x7fc00000);
            r.prefix_ok = true;
            r.whole = i + k == len;
            return r;
        }
        return r;  // no number
    }
    if (i + 1 < len && p[i] == '0' && lower(p[i + 1]) == 'x') {
        r.fatal = kFatalHex;
        return r;
    }
    // mantissa: the first 19 significant digits in w, the rest counted
    const uint32_t mant = i;
    uint64_t w = 0;
    int nsig = 0, nkept = 0;
    long long dexp = 0;  // decimal exponent adjustment of w
    bool trunc = false, any_digit = false, seen_dot = false;
    for (; i < len; ++i) {
        const uint32_t c = p[i];
        if (is_digit(c)) {
            any_digit = true;
            const uint32_t d = c - '0';
            if (nsig == 0 && d == 0) {  // leading zero
                if (seen_dot) --dexp;
                continue;
            }
            ++nsig;
            if (nkept < 19) {
                w = w * 10 + d;
                ++nkept;
                if (seen_dot) --dexp;
            } else {
                if (d) trunc = true;
                if (!seen_dot) ++dexp;
            }
        } else if (c == '.' && !seen_dot) {
            seen_dot = true;
        } else {
            break;
        }
    }
    if (!any_digit) return r;  // "", "+", ".", "-." ...
    r.prefix_ok = true;
    // exponent: glibc's fscanf consumes "e[sign]digits"; an 'e' (and sign)
    // without digits is consumed too and leaves the mantissa's value
    long long ex = 0;
    if (i < len && lower(p[i]) == 'e') {
        uint32_t j = i + 1;
        bool eneg = false;
        if (j < len && (p[j] == '+' || p[j] == '-')) eneg = p[j++] == '-';
        for (; j < len && is_digit(p[j]); ++j)
            if (ex < 100000) ex = ex * 10 + (p[j] - '0');
        if (eneg) ex = -ex;
        i = j;
    }
    r.whole = i == len;
    double d;
    if (nsig == 0) {
        d = 0.0;
    } else {
        const long long q = dexp + ex;  // value = w * 10^q (w holds nkept digits)
        if (!trunc && w <= (1ull << 53) && q >= -22 && q <= 22) {
            // Clinger: w and 10^|q| are exact doubles, one IEEE operation
            constexpr double p10[23] = {1e0,  1e1,  1e2,  1e3,  1e4,  1e5,  1e6,  1e7,  1e8,  1e9,  1e10, 1e11,
                                        1e12, 1e13, 1e14, 1e15, 1e16, 1e17, 1e18, 1e19, 1e20, 1e21, 1e22};
            d = q >= 0 ? __dmul_rn((double)w, p10[q]) : __ddiv_rn((double)w, p10[-q]);
        } else {
            // magnitude: value in [10^(mag-1), 10^mag)
            const long long mag = (long long)nkept + q;
            if (mag > 39) {
                d = __longlong_as_double(0x7ff0000000000000ll);  // rounds to FP32 infinity
            } else if (mag < -47) {
                d = 0.0;  // below half the smallest FP32 subnormal
            } else if (nsig > kMaxSigDigits) {
                r.fatal = kFatalDigits;
                return r;
            } else {
                // all significant digits: value = D * 10^(q + nkept - nsig)
                d = exact_decimal(p + mant, nsig, (int)(q + nkept - nsig));
            }
        }
    }
    const float f = __double2float_rn(d);
    r.value = neg ? -f : f;
    return r;
}

struct ParseArgs {
    const uint8_t *buf;
    uint64_t len;
    const uint64_t *chunk_base;
    uint32_t nmodes;
    uint64_t hdr;   // header tokens: nmodes + 1
    uint64_t nrec;  // nonzeros with all N+1 tokens present
    uint32_t start_index;
    uint32_t *inds[kMaxModes];
    float *vals;
    ParseSlots *slots;
};

__global__ void __launch_bounds__(kIngThreads) tok_parse_kernel(ParseArgs a)
{
    __shared__ uint32_t s_warp[kIngThreads / 32];
    const uint64_t base = (uint64_t)blockIdx.x * kIngChunk;
    uint64_t ord = a.chunk_base[blockIdx.x];
    const uint32_t F = a.nmodes + 1;
    for (int j = 0; j < kIngSteps; ++j) {
        const uint64_t off = base + (uint64_t)j * kIngStep + threadIdx.x * kIngSeg;
        uint32_t starts = seg_starts(a.buf, off);
        uint32_t total;
        const uint32_t before = block_exclusive_scan<uint32_t>(__popc(starts), s_warp, total);
        uint64_t t = ord + before;
        while (starts) {
            const int b = __ffs(starts) - 1;
            starts &= starts - 1;
            const uint64_t pos = off + b;
            const uint64_t tok = t++;
            if (tok < a.hdr) continue;  // header, read on the host
            const uint8_t *p = a.buf + pos;
            uint32_t len = 0;
            while (len < kMaxToken && pos + len < a.len && !is_ws(p[len])) ++len;
            const uint64_t u = tok - a.hdr;
            const uint64_t rec = u / F;
            const uint32_t field = (uint32_t)(u - rec * F);
            if (len == kMaxToken) {
                atomicMin(&a.slots->fatal, (unsigned long long)tok);
                atomicOr(&a.slots->fatal_flags, kFatalLong);
                continue;
            }
            if (field < a.nmodes) {
                const IndexTok x = parse_index(p, len);
                if (!x.whole) atomicMin(&a.slots->bad, (unsigned long long)tok * 2);
                if (x.prefix_ok && x.value < a.start_index) atomicMin(&a.slots->low, (unsigned long long)tok);
                if (rec < a.nrec) a.inds[field][rec] = x.value - a.start_index;
            } else {
                const ValueTok v = parse_value(p, len);
                if (v.fatal) {
                    atomicMin(&a.slots->fatal, (unsigned long long)tok);
                    atomicOr(&a.slots->fatal_flags, v.fatal);
                    continue;
                }
                if (!v.whole) atomicMin(&a.slots->bad, (unsigned long long)tok * 2 + (v.prefix_ok ? 1 : 0));
                if (rec < a.nrec) a.vals[rec] = v.value;
            }
        }
        ord += total;
    }
}

// FP64 values of a binary file (4-byte aligned) rounded to FP32.
__global__ void f64_to_f32_kernel(const uint32_t *src, uint64_t n, float *dst)
{
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t bits = (uint64_t)src[2 * i] | ((uint64_t)src[2 * i + 1] << 32);
        dst[i] = __double2float_rn(__longlong_as_double((long long)bits));
    }
}

// ---------------------------------------------------------------------------
// Duplicate merge
// ---------------------------------------------------------------------------
__global__ void gather_key_kernel(const uint32_t *ind, const uint32_t *perm, uint64_t n, uint64_t *key)
{
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        key[i] = ind[perm[i]];
}

__global__ void iota_kernel(uint32_t *v, uint64_t n)
{
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        v[i] = (uint32_t)i;
}

struct DedupArgs {
    uint32_t nmodes;
    uint64_t n;
    const uint32_t *perm;
    const uint32_t *inds[kMaxModes];
    const float *vals;
};

__device__ __forceinline__ bool run_head(const DedupArgs &a, uint64_t i)
{
    if (i == 0) return true;
    const uint32_t p = a.perm[i], q = a.perm[i - 1];
    for (uint32_t m = 0; m < a.nmodes; ++m)
        if (a.inds[m][p] != a.inds[m][q]) return true;
    return false;
}

struct HeadIn {
    DedupArgs a;
    __device__ uint64_t operator()(uint64_t i) const { return run_head(a, i) ? 1 : 0; }
};
struct HeadOut {
    DedupArgs a;
    uint32_t *out_inds[kMaxModes];
    float *out_vals;
    __device__ void operator()(uint64_t i, uint64_t prefix, uint64_t head) const
    {
        if (!head) return;
        const uint32_t p = a.perm[i];
        for (uint32_t m = 0; m < a.nmodes; ++m) out_inds[m][prefix] = a.inds[m][p];
        float s = a.vals[p];
        for (uint64_t j = i + 1; j < a.n && !run_head(a, j); ++j) s = __fadd_rn(s, a.vals[a.perm[j]]);
        out_vals[prefix] = s;
    }
};

unsigned grid_for_n(uint64_t n)
{
    return (unsigned)std::max<uint64_t>(1, std::min<uint64_t>((n + 255) / 256, (uint64_t)sm_count() * 8));
}

int bits_for(uint32_t maxval)
{
    int b = 0;
    while (b < 32 && (maxval >> b)) ++b;
    return b;
}

}  // namespace

// Sorts the nonzeros of t by coordinate and merges repeated coordinates.
int dedupe_coo(ptiB200Tensor *t, cudaStream_t s)
{
    const char *mod = "B200 SpTns Load";
    const uint64_t n = t->nnz;
    if (n <= 1) return 0;
    PTI_CHECK(n < 0xFFFFFFFFull, PTIERR_VALUE_ERROR, mod, "too many nonzeros to merge");
    DevBuf keys, perm;
    RadixScratch sc;
    PTI_CUDA(keys.alloc(padded(n * 8), s), mod);
    PTI_CUDA(perm.alloc(padded(n * 4), s), mod);
    PTI_TRY(sc.alloc(n, s));
    iota_kernel<<<grid_for_n(n), 256, 0, s>>>(perm.as<uint32_t>(), n);
    // LSD over the modes: the last mode first, mode 0 last (most significant)
    for (int m = (int)t->nmodes - 1; m >= 0; --m) {
        gather_key_kernel<<<grid_for_n(n), 256, 0, s>>>(t->inds[m].as<uint32_t>(), perm.as<uint32_t>(), n,
                                                        keys.as<uint64_t>());
        const int nbits = bits_for(t->ndims[m] ? t->ndims[m] - 1 : 0);
        PTI_TRY(radix_sort_pairs(keys, perm, n, ((nbits + 7) / 8) * 8, sc, s));
    }
    DedupArgs a;
    a.nmodes = t->nmodes;
    a.n = n;
    a.perm = perm.as<uint32_t>();
    for (uint32_t m = 0; m < t->nmodes; ++m) a.inds[m] = t->inds[m].as<uint32_t>();
    a.vals = t->vals.as<float>();
    DevBuf out_inds[kMaxModes], out_vals, tmp;
    HeadOut ho;
    ho.a = a;
    for (uint32_t m = 0; m < t->nmodes; ++m) {
        PTI_CUDA(out_inds[m].alloc(padded(n * 4), s), mod);
        ho.out_inds[m] = out_inds[m].as<uint32_t>();
    }
    PTI_CUDA(out_vals.alloc(padded(n * 4), s), mod);
    ho.out_vals = out_vals.as<float>();
    PTI_CUDA(tmp.alloc(padded(scan_tmp_elems<uint64_t>(n) * 8), s), mod);
    uint64_t uniq = 0;
    PTI_TRY((exclusive_scan<uint64_t>(HeadIn{a}, ho, n, tmp.as<uint64_t>(), &uniq, s)));
    for (uint32_t m = 0; m < t->nmodes; ++m) t->inds[m].swap(out_inds[m]);
    t->vals.swap(out_vals);
    t->nnz = uniq;
    return 0;
}

namespace {

// Pinned staging for file reads, kept for the life of the process: kReaders
// reader threads with two kReadChunk buffers each, every thread with its own
// stream and an event per buffer.  Loads are serialised on its mutex.
constexpr int kReaders = 4;
struct ReadPool {
    std::mutex mu;
    bool ready = false;
    unsigned char *pin[kReaders][2] = {};
    cudaStream_t st[kReaders] = {};
    cudaEvent_t ev[kReaders][2] = {};
};
ReadPool &read_pool(int dev)
{
    static ReadPool p[64];  // per device: the streams and events belong to one
    return p[dev & 63];
}

// Reads the whole file into a device buffer padded with spaces to
// `pad_to`-byte multiples (+64).  kReaders threads pread interleaved chunks
// of kReadChunk bytes into pinned buffers (two per thread) and copy each to
// its place on the device on their own streams, so reading the page cache,
// which one thread cannot do at link speed, runs in parallel and overlaps
// the copies.
int read_to_device(const char *fname, DevBuf &dbuf, uint64_t &len, std::vector<unsigned char> &head,
                   size_t head_bytes, uint64_t pad_to, cudaStream_t s)
{
    const char *mod = "B200 SpTns Load";
    const int fd = open(fname, O_RDONLY);
    PTI_CHECK(fd >= 0, PTIERR_OS_ERROR + errno, mod, std::strerror(errno));
    struct stat stbuf;
    if (fstat(fd, &stbuf) != 0) {
        const int e = errno;
        close(fd);
        PTI_FAIL(PTIERR_OS_ERROR + e, mod, "cannot size the file");
    }
    len = (uint64_t)stbuf.st_size;
    int dev = 0;
    cudaGetDevice(&dev);
    ReadPool &P = read_pool(dev);
    std::lock_guard<std::mutex> lock(P.mu);
    cudaError_t ce = cudaSuccess;
    if (!P.ready) {
        for (int t = 0; t < kReaders && ce == cudaSuccess; ++t) {
            ce = cudaStreamCreateWithFlags(&P.st[t], cudaStreamNonBlocking);
            for (int b = 0; b < 2 && ce == cudaSuccess; ++b) {
                ce = cudaHostAlloc(reinterpret_cast<void **>(&P.pin[t][b]), kReadChunk, cudaHostAllocDefault);
                if (ce == cudaSuccess) ce = cudaEventCreateWithFlags(&P.ev[t][b], cudaEventDisableTiming);
            }
        }
        if (ce != cudaSuccess) {
            close(fd);
            PTI_CUDA(ce, mod);
        }
        P.ready = true;
    }
    const uint64_t alloc = std::max<uint64_t>(1, (len + pad_to - 1) / pad_to) * pad_to + 64;
    cudaEvent_t filled = nullptr;
    ce = dbuf.alloc(alloc, s);
    if (ce == cudaSuccess) ce = cudaMemsetAsync(dbuf.ptr, ' ', alloc, s);
    if (ce == cudaSuccess) ce = cudaEventCreateWithFlags(&filled, cudaEventDisableTiming);
    if (ce == cudaSuccess) ce = cudaEventRecord(filled, s);
    if (ce != cudaSuccess) {
        close(fd);
        if (filled) cudaEventDestroy(filled);
        PTI_CUDA(ce, mod);
    }
    head.assign(std::min<uint64_t>(head_bytes, len), 0);
    const uint64_t nchunks = (len + kReadChunk - 1) / kReadChunk;
    const int nthreads = (int)std::min<uint64_t>(kReaders, std::max<uint64_t>(nchunks, 1));
    std::vector<int> err(nthreads, 0);
    std::vector<cudaError_t> cerr(nthreads, cudaSuccess);
    auto reader = [&](int t) {
        cudaError_t c = cudaSetDevice(dev);
        if (c == cudaSuccess) c = cudaStreamWaitEvent(P.st[t], filled, 0);  // after the fill with spaces
        int slot = 0;
        for (uint64_t k = t; c == cudaSuccess && k < nchunks; k += nthreads, slot ^= 1) {
            c = cudaEventSynchronize(P.ev[t][slot]);  // the buffer's previous copy has landed
            if (c != cudaSuccess) break;
            const uint64_t off = k * kReadChunk;
            const size_t want = (size_t)std::min<uint64_t>(kReadChunk, len - off);
            size_t got = 0;
            while (got < want) {
                const ssize_t r = pread(fd, P.pin[t][slot] + got, want - got, (off_t)(off + got));
                if (r <= 0) break;
                got += (size_t)r;
            }
            if (got != want) {
                err[t] = EIO;
                break;
            }
            if (off < head.size())
                std::memcpy(head.data() + off, P.pin[t][slot], std::min<uint64_t>(want, head.size() - off));
            c = cudaMemcpyAsync(dbuf.as<unsigned char>() + off, P.pin[t][slot], want, cudaMemcpyHostToDevice,
                                P.st[t]);
            if (c == cudaSuccess) c = cudaEventRecord(P.ev[t][slot], P.st[t]);
        }
        if (c == cudaSuccess) c = cudaStreamSynchronize(P.st[t]);
        cerr[t] = c;
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < nthreads; ++t) pool.emplace_back(reader, t);
    reader(0);
    for (auto &th : pool) th.join();
    close(fd);
    cudaEventDestroy(filled);
    for (int t = 0; t < nthreads; ++t) {
        PTI_CHECK(!err[t], PTIERR_OS_ERROR + err[t], mod, "short read");
        PTI_CUDA(cerr[t], mod);
    }
    return 0;
}

// fscanf("%u") on the header: skips white space, reads one number.
bool header_uint(const std::vector<unsigned char> &h, size_t &pos, uint32_t &out)
{
    while (pos < h.size() && (h[pos] == ' ' || (h[pos] >= 9 && h[pos] <= 13))) ++pos;
    bool neg = false;
    if (pos < h.size() && (h[pos] == '+' || h[pos] == '-')) neg = h[pos++] == '-';
    uint64_t v = 0;
    bool over = false;
    const size_t d0 = pos;
    for (; pos < h.size() && h[pos] >= '0' && h[pos] <= '9'; ++pos) {
        const uint64_t d = h[pos] - '0';
        if (v > (~0ull - d) / 10) over = true;
        else v = v * 10 + d;
    }
    if (pos == d0) return false;
    out = over ? 0xFFFFFFFFu : (uint32_t)(neg ? 0ull - v : v);
    return true;
}

int parse_text(ptiB200Tensor *t, uint32_t start_index, const DevBuf &dbuf, uint64_t len,
               const std::vector<unsigned char> &head, cudaStream_t s)
{
    const char *mod = "B200 SpTns Load";
    size_t pos = 0;
    uint32_t nm = 0;
    PTI_CHECK(header_uint(head, pos, nm), PTIERR_VALUE_ERROR, mod, "missing number of modes");
    PTI_CHECK(nm >= 1 && nm <= (uint32_t)kMaxModes, PTIERR_VALUE_ERROR, mod, "unsupported number of modes");
    t->nmodes = nm;
    t->ndims.assign(nm, 0);
    for (uint32_t m = 0; m < nm; ++m)
        PTI_CHECK(header_uint(head, pos, t->ndims[m]), PTIERR_VALUE_ERROR, mod, "bad mode sizes");
    // A last mode size with characters glued to it: fscanf stops at them, so
    // there are no nonzeros.
    const bool glued = pos < head.size() && !(head[pos] == ' ' || (head[pos] >= 9 && head[pos] <= 13));
    if (glued) {
        for (uint32_t m = 0; m < nm; ++m) PTI_CUDA(t->inds[m].alloc(padded(0), s), mod);
        PTI_CUDA(t->vals.alloc(padded(0), s), mod);
        t->nnz = 0;
        return 0;
    }

    const uint64_t nchunks = std::max<uint64_t>(1, (len + kIngChunk - 1) / kIngChunk);
    DevBuf counts, bases, tmp, slots;
    PTI_CUDA(counts.alloc(padded(nchunks * 4), s), mod);
    PTI_CUDA(bases.alloc(padded(nchunks * 8), s), mod);
    PTI_CUDA(tmp.alloc(padded(scan_tmp_elems<uint64_t>(nchunks) * 8), s), mod);
    PTI_CUDA(slots.alloc(padded(sizeof(ParseSlots)), s), mod);
    tok_count_kernel<<<(unsigned)nchunks, kIngThreads, 0, s>>>(dbuf.as<uint8_t>(), counts.as<uint32_t>());
    uint64_t ntok = 0;
    PTI_TRY((exclusive_scan<uint64_t>(CountIn{counts.as<uint32_t>()}, OffsetOut{bases.as<uint64_t>()}, nchunks,
                                      tmp.as<uint64_t>(), &ntok, s)));
    const uint64_t hdr = (uint64_t)nm + 1;
    PTI_CHECK(ntok >= hdr, PTIERR_VALUE_ERROR, mod, "bad mode sizes");
    const uint64_t nrec = (ntok - hdr) / hdr;

    for (uint32_t m = 0; m < nm; ++m) PTI_CUDA(t->inds[m].alloc(padded(nrec * 4), s), mod);
    PTI_CUDA(t->vals.alloc(padded(nrec * 4), s), mod);
    ParseSlots init{~0ull, ~0ull, ~0ull, 0u, 0u};
    PTI_CUDA(cudaMemcpyAsync(slots.ptr, &init, sizeof init, cudaMemcpyHostToDevice, s), mod);
    ParseArgs a{};
    a.buf = dbuf.as<uint8_t>();
    a.len = len;
    a.chunk_base = bases.as<uint64_t>();
    a.nmodes = nm;
    a.hdr = hdr;
    a.nrec = nrec;
    a.start_index = start_index;
    for (uint32_t m = 0; m < nm; ++m) a.inds[m] = t->inds[m].as<uint32_t>();
    a.vals = t->vals.as<float>();
    a.slots = slots.as<ParseSlots>();
    tok_parse_kernel<<<(unsigned)nchunks, kIngThreads, 0, s>>>(a);
    PTI_CUDA(cudaGetLastError(), mod);
    ParseSlots r;
    PTI_CUDA(cudaMemcpyAsync(&r, slots.ptr, sizeof r, cudaMemcpyDeviceToHost, s), mod);
    PTI_CUDA(cudaStreamSynchronize(s), mod);

    // Where fscanf stops: before the first malformed token's nonzero, or
    // after it when that token is a value with a number in front.
    uint64_t nnz = nrec, stop = ~0ull;
    if (r.bad != ~0ull) {
        stop = r.bad >> 1;
        const uint64_t u = stop - hdr, rec = u / hdr, field = u % hdr;
        const uint64_t cut = (field == nm && (r.bad & 1)) ? rec + 1 : rec;
        nnz = std::min(nnz, cut);
    }
    if (r.fatal != ~0ull && r.fatal < stop) {
        const char *why = (r.fatal_flags & kFatalHex)          ? "hexadecimal values are not supported"
                          : (r.fatal_flags & kFatalNanPayload) ? "nan(...) values are not supported"
                          : (r.fatal_flags & kFatalLong)       ? "token longer than 4096 bytes"
                                                               : "value with more than 100 significant digits";
        PTI_FAIL(PTIERR_VALUE_ERROR, mod, why);
    }
    // src/sptensor/load.c:94-96: an index read below start_index is an error
    PTI_CHECK(r.low == ~0ull || r.low > stop, PTIERR_VALUE_ERROR, mod, "index < start_index");
    t->nnz = nnz;
    return 0;
}

int parse_binary(ptiB200Tensor *t, const DevBuf &dbuf, uint64_t len, const std::vector<unsigned char> &head,
                 cudaStream_t s)
{
    const char *mod = "B200 SpTns Load";
    // {int32 magic, u64 idx_width, u64 val_width}, nmodes, dims, nnz (idx_width
    // each), the index arrays mode by mode, the values (src/sptensor/load.c:120-265)
    PTI_CHECK(head.size() >= 24, PTIERR_VALUE_ERROR, mod, "truncated header");
    uint64_t iw, vw;
    std::memcpy(&iw, head.data() + 4, 8);
    std::memcpy(&vw, head.data() + 12, 8);
    PTI_CHECK(iw == 4, PTIERR_VALUE_ERROR, mod, "only 32-bit indices are supported");
    PTI_CHECK(vw == 4 || vw == 8, PTIERR_VALUE_ERROR, mod, "bad value width");
    uint32_t nm;
    std::memcpy(&nm, head.data() + 20, 4);
    PTI_CHECK(nm >= 1 && nm <= (uint32_t)kMaxModes, PTIERR_VALUE_ERROR, mod, "unsupported number of modes");
    const size_t dims_end = 24 + 4ull * nm + 4;
    PTI_CHECK(head.size() >= dims_end, PTIERR_VALUE_ERROR, mod, "truncated header");
    t->nmodes = nm;
    t->ndims.assign(nm, 0);
    std::memcpy(t->ndims.data(), head.data() + 24, 4ull * nm);
    uint32_t nnz32;
    std::memcpy(&nnz32, head.data() + 24 + 4ull * nm, 4);
    const uint64_t nnz = nnz32;
    PTI_CHECK(len >= dims_end + nnz * (4ull * nm + vw), PTIERR_VALUE_ERROR, mod, "truncated file");
    t->nnz = nnz;
    const unsigned char *src = dbuf.as<unsigned char>() + dims_end;
    for (uint32_t m = 0; m < nm; ++m) {
        PTI_CUDA(t->inds[m].alloc(padded(nnz * 4), s), mod);
        if (nnz) PTI_CUDA(cudaMemcpyAsync(t->inds[m].ptr, src + 4ull * m * nnz, nnz * 4, cudaMemcpyDeviceToDevice, s),
                          mod);
    }
    PTI_CUDA(t->vals.alloc(padded(nnz * 4), s), mod);
    const unsigned char *vsrc = src + 4ull * nm * nnz;
    if (nnz && vw == 4) PTI_CUDA(cudaMemcpyAsync(t->vals.ptr, vsrc, nnz * 4, cudaMemcpyDeviceToDevice, s), mod);
    if (nnz && vw == 8)
        f64_to_f32_kernel<<<grid_for_n(nnz), 256, 0, s>>>(reinterpret_cast<const uint32_t *>(vsrc), nnz,
                                                          t->vals.as<float>());
    PTI_CUDA(cudaGetLastError(), mod);
    return 0;
}

}  // namespace

// Loads a .tns/.coo (text) or .bin (SPLATT binary) file into t's COO arrays;
// `text` receives which parser ran.
int ingest_file(ptiB200Tensor *t, uint32_t start_index, const char *fname, bool *text, cudaStream_t s)
{
    const char *mod = "B200 SpTns Load";
    PTI_CHECK(fname, PTIERR_VALUE_ERROR, mod, "null file name");
    configure_pool_once();
    cudaGetDevice(&t->device);
    t->hicoo = false;
    // File type by extension (src/sptensor/load.c:25-60): .bin is binary,
    // .tns and .coo are text, anything else is read as text with a warning.
    const char *suffix = std::strrchr(fname, '.');
    const bool binary = suffix && std::strcmp(suffix, ".bin") == 0;
    if (!binary && !(suffix && (std::strcmp(suffix, ".tns") == 0 || std::strcmp(suffix, ".coo") == 0)) &&
        !std::getenv("HIPARTI_B200_QUIET"))
        std::fprintf(stderr, "extension for '%s' not recognized; reading it as a text coordinate file\n", fname);
    if (text) *text = !binary;
    DevBuf dbuf;
    uint64_t len = 0;
    std::vector<unsigned char> head;
    PTI_TRY(read_to_device(fname, dbuf, len, head, binary ? 24 + 4 * kMaxModes + 8 : 4096, kIngChunk, s));
    if (binary) PTI_TRY(parse_binary(t, dbuf, len, head, s));
    else PTI_TRY(parse_text(t, start_index, dbuf, len, head, s));
    PTI_CUDA(cudaStreamSynchronize(s), mod);
    return 0;
}

}  // namespace pti

extern "C" {

int ptiB200LoadSparseTensor(ptiB200Tensor **out, ptiIndex start_index, const char *fname, int dedupe, void *stream)
{
    using namespace pti;
    const char *mod = "B200 SpTns Load";
    PTI_CHECK(out && fname, PTIERR_VALUE_ERROR, mod, "null argument");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    auto *t = new ptiB200Tensor();
    int r = ingest_file(t, start_index, fname, nullptr, s);
    if (!r && t->nmodes < 2) r = complain(mod, PTIERR_VALUE_ERROR, __FILE__, __LINE__, "a device tensor needs two or more modes");
    if (!r && dedupe) r = dedupe_coo(t, s);
    // the MTTKRP kernels index factor rows with these: they must fit the modes
    if (!r) r = check_coo_ranges(t, s);
    if (!r && cudaStreamSynchronize(s) != cudaSuccess)
        r = complain(mod, PTIERR_CUDA_ERROR, __FILE__, __LINE__, "stream synchronisation failed");
    if (r) {
        delete t;
        return r;
    }
    *out = t;
    return 0;
}

int ptiB200DownloadCOO(ptiB200Tensor const *t, ptiIndex * const *inds, ptiValue *vals)
{
    using namespace pti;
    const char *mod = "B200 Download";
    PTI_CHECK(t && !t->hicoo, PTIERR_VALUE_ERROR, mod, "not a device COO tensor");
    cudaStream_t s = sync_stream();
    for (uint32_t m = 0; m < t->nmodes && t->nnz; ++m)
        if (inds && inds[m])
            PTI_CUDA(cudaMemcpyAsync(inds[m], t->inds[m].ptr, t->nnz * 4, cudaMemcpyDeviceToHost, s), mod);
    if (vals && t->nnz) PTI_CUDA(cudaMemcpyAsync(vals, t->vals.ptr, t->nnz * 4, cudaMemcpyDeviceToHost, s), mod);
    PTI_CUDA(cudaStreamSynchronize(s), mod);
    return 0;
}

}  // extern "C"
