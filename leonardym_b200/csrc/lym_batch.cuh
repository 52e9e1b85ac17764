// Multi-right-hand-side (batched) fields and kernels.
//
// A batch holds nb right-hand sides (nb a power of two, 2 <= nb <= 32) of one parity.
// The RHS are taken in pairs (2q, 2q+1), q < np = nb / 2, and a pair is the unit of
// work of one thread: every arithmetic step runs on float2 registers whose two lanes
// are the two RHS of the pair, with the packed FP32 instructions of sm_100
// (__ffma2_rn / __fadd2_rn / __fmul2_rn, sub.rn.f32x2), which halves the issued
// arithmetic.
//
// Storage, with the pair index innermost so that the np threads of a half-site read
// consecutive 16-byte words:
//   FP32: float4 v[(c * stride + h) * np + q] = (re_2q, re_2q+1, im_2q, im_2q+1)
//         for complex component c = spin * 3 + colour (12 per site);
//   FP16: int4 v[(w * stride + h) * np + q] = halves (re_a, re_b, im_a, im_b) of
//         component 2w followed by those of component 2w+1 (w < 6), and a float2
//         norm n[h * np + q] = (max |.| of RHS 2q, of RHS 2q+1).
// Link, clover and neighbour-index words of a half-site are read by all np threads
// of that half-site (broadcast), so their bytes are shared by the whole batch; the
// links are read in the 12-real format or, for SU(3), in all 18 reals (GaugeF18P), and
// expanded in registers.
#pragma once

#include <type_traits>

#include "lym_blas.cuh"
#include "lym_dslash.cuh"

namespace lym {

constexpr int kMaxBatch = 32;
constexpr int kBatchMaxRed = 8;  // FP64 reductions per RHS a batched vector kernel may carry

// ------------------------------------------------------- pair arithmetic ---
struct c2 {  // one complex component of the two RHS of a pair
    float2 re, im;
};

LYM_D float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
LYM_D float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
LYM_D float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
LYM_D float2 sub2(float2 a, float2 b)  // a - b in one packed instruction (no negated copy of b)
{
    float2 d;
    asm("{\n\t.reg .b64 ra, rb, rd;\n\t"
        "mov.b64 ra, {%2, %3};\n\t"
        "mov.b64 rb, {%4, %5};\n\t"
        "sub.rn.f32x2 rd, ra, rb;\n\t"
        "mov.b64 {%0, %1}, rd;\n\t}"
        : "=f"(d.x), "=f"(d.y)
        : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
    return d;
}

// a + s * code * z with code 0: +1, 1: -1, 2: +i, 3: -i (s = +1 or -1, compile time)
template <int S> LYM_D c2 add_code(c2 a, int code, c2 z)
{
    const bool plus = (S > 0) == (code == 0 || code == 3);
    switch (code) {
    case 0:
    case 1: return plus ? c2{add2(a.re, z.re), add2(a.im, z.im)} : c2{sub2(a.re, z.re), sub2(a.im, z.im)};
    case 2:  // +i z = (-z.im, z.re)
        return S > 0 ? c2{sub2(a.re, z.im), add2(a.im, z.re)} : c2{add2(a.re, z.im), sub2(a.im, z.re)};
    default:  // -i z = (z.im, -z.re)
        return S > 0 ? c2{add2(a.re, z.im), sub2(a.im, z.re)} : c2{sub2(a.re, z.im), add2(a.im, z.re)};
    }
}

// ----------------------------------------------------- asynchronous copies --
LYM_D unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }
LYM_D void cp_async16(unsigned saddr, const void *g)
{
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(saddr), "l"(g) : "memory");
}
LYM_D void cp_async8(unsigned saddr, const void *g)
{
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(saddr), "l"(g) : "memory");
}
LYM_D void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N> LYM_D void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// Bulk copies (cp.async.bulk, this GPU's global memory -> this CTA's shared memory, no
// multicast) completing on an mbarrier in shared memory.
LYM_D void mbar_init(unsigned mb)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(mb) : "memory");
}
LYM_D void mbar_init_fence() { asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory"); }
LYM_D void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }
LYM_D void mbar_expect(unsigned mb, unsigned bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(mb), "r"(bytes) : "memory");
}
LYM_D void bulk_copy(unsigned dst, const void *src, unsigned bytes, unsigned mb)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(dst),
                 "l"(src), "r"(bytes), "r"(mb)
                 : "memory");
}
// waits for the phase of the given parity; gives up after a bounded number of polls (a
// copy that never lands must not hang the GPU) and returns whether the phase completed
LYM_D bool mbar_wait(unsigned mb, unsigned parity)
{
    for (int it = 0; it < (1 << 16); ++it) {
        unsigned done;
        asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                     "selp.u32 %0, 1, 0, p;\n\t}"
                     : "=r"(done)
                     : "r"(mb), "r"(parity)
                     : "memory");
        if (done) return true;
    }
    return false;
}

// ------------------------------------------------------------- batch views --
// One RHS r of a FP32 pair-layout batch, as a single half-spinor view (slot set-up,
// extraction and reliable updates; not on the iteration path).  A 16-byte word holds
// component c of both RHS of the pair (re_a, re_b, im_a, im_b), so the words of one RHS
// lie 16 << lognp bytes apart: reads take the whole word (one request per word instead
// of one per float).
struct SlotF {
    float *f;
    int stride, lognp, r;
    static constexpr bool kPerComponent = true;  // get / put one component at a time
    LYM_HD SlotF par(int) const { return *this; }
    LYM_D size_t base(int c, int h) const
    {
        return (((((size_t)c * stride + h) << lognp) + (r >> 1)) << 2) + (r & 1);
    }
    LYM_D size_t word_at(int c, int h) const { return (((size_t)c * stride + h) << lognp) + (r >> 1); }
    // the word of component c at half-site h (this RHS and its pair mate)
    LYM_D float4 word(int c, int h) const { return reinterpret_cast<const float4 *>(f)[word_at(c, h)]; }
    LYM_D cx<double> lane(float4 w) const
    {
        return (r & 1) ? cx<double>{(double)w.y, (double)w.w} : cx<double>{(double)w.x, (double)w.z};
    }
    // w with this RHS's value replaced by s rounded to FP32; the mate's floats unchanged
    LYM_D float4 with(float4 w, cx<double> s) const
    {
        if (r & 1) {
            w.y = (float)s.re;
            w.w = (float)s.im;
        } else {
            w.x = (float)s.re;
            w.z = (float)s.im;
        }
        return w;
    }
    // writes a whole word back: only where nothing else writes the mate's lane meanwhile
    LYM_D void put_word(int c, int h, float4 w) const { reinterpret_cast<float4 *>(f)[word_at(c, h)] = w; }
    LYM_D cx<double> get(int c, int h) const { return lane(word(c, h)); }
    LYM_D void put(int c, int h, cx<double> s) const
    {
        const size_t b = base(c, h);
        f[b] = (float)s.re;
        f[b + 2] = (float)s.im;
    }
    template <typename R> LYM_D void load(int h, cx<R> s[12]) const
    {
#pragma unroll
        for (int c = 0; c < 12; ++c) {
            const cx<double> v = get(c, h);
            s[c] = cx<R>{(R)v.re, (R)v.im};
        }
    }
    template <typename R> LYM_D void store(int h, const cx<R> s[12]) const
    {
#pragma unroll
        for (int c = 0; c < 12; ++c) {
            const size_t b = base(c, h);
            f[b] = (float)s[c].re;
            f[b + 2] = (float)s[c].im;
        }
    }
};

struct BatchF {
    float4 *v;
    int stride, lognp;
    // word index; a batch holds at most 2^32 words (checked when it is allocated)
    LYM_D unsigned at(int c, int h, int q) const { return (((unsigned)c * stride + h) << lognp) + q; }
    LYM_D void load(int h, int q, c2 x[12]) const
    {
        const unsigned b = at(0, h, q), s = (unsigned)stride << lognp;
#pragma unroll
        for (int c = 0; c < 12; ++c) {
            const float4 w = __ldg(v + b + c * s);
            x[c] = c2{make_float2(w.x, w.y), make_float2(w.z, w.w)};
        }
    }
    // streaming read (a field read once per launch)
    LYM_D void load_cs(int h, int q, c2 x[12]) const
    {
        const unsigned b = at(0, h, q), s = (unsigned)stride << lognp;
#pragma unroll
        for (int c = 0; c < 12; ++c) {
            const float4 w = __ldcs(v + b + c * s);
            x[c] = c2{make_float2(w.x, w.y), make_float2(w.z, w.w)};
        }
    }
    LYM_D void store(int h, int q, const c2 x[12]) const
    {
        const unsigned b = at(0, h, q), s = (unsigned)stride << lognp;
#pragma unroll
        for (int c = 0; c < 12; ++c) __stcs(v + b + c * s, make_float4(x[c].re.x, x[c].re.y, x[c].im.x, x[c].im.y));
    }
    // component c of both RHS of the pair in FP64 (vector algebra, one word at a time)
    LYM_D void get(int h, int q, int c, cx<double> &a, cx<double> &b) const
    {
        const float4 w = __ldg(v + at(c, h, q));
        a = cx<double>{(double)w.x, (double)w.z};
        b = cx<double>{(double)w.y, (double)w.w};
    }
    LYM_D void put(int h, int q, int c, cx<double> a, cx<double> b) const
    {
        v[at(c, h, q)] = make_float4((float)a.re, (float)b.re, (float)a.im, (float)b.im);
    }
    // FP64 values of both RHS of the pair (vector algebra)
    LYM_D void load_d(int h, int q, cx<double> a[12], cx<double> b[12]) const
    {
#pragma unroll
        for (int c = 0; c < 12; ++c) {
            const float4 w = __ldg(v + at(c, h, q));
            a[c] = cx<double>{(double)w.x, (double)w.z};
            b[c] = cx<double>{(double)w.y, (double)w.w};
        }
    }
    LYM_D void store_d(int h, int q, const cx<double> a[12], const cx<double> b[12]) const
    {
#pragma unroll
        for (int c = 0; c < 12; ++c)
            v[at(c, h, q)] = make_float4((float)a[c].re, (float)b[c].re, (float)a[c].im, (float)b[c].im);
    }
    // asynchronous copy of the pair's 12 words into shared memory (word c at s0 + c * sstep
    // bytes) and the read back from there (word c at p0[c * step])
    LYM_D void stage(unsigned s0, unsigned sstep, int h, int q) const
    {
        const unsigned b = at(0, h, q), s = (unsigned)stride << lognp;
#pragma unroll
        for (int c = 0; c < 12; ++c) cp_async16(s0 + c * sstep, v + b + c * s);
    }
    LYM_D void unstage(const float4 *p0, int step, c2 x[12]) const
    {
#pragma unroll
        for (int c = 0; c < 12; ++c) {
            const float4 w = p0[c * step];
            x[c] = c2{make_float2(w.x, w.y), make_float2(w.z, w.w)};
        }
    }
    // the 6 components of spin block blk (spins 0, 1 or 2, 3)
    LYM_D void unstage_block(const float4 *p0, int step, int blk, c2 x[6]) const
    {
#pragma unroll
        for (int c = 0; c < 6; ++c) {
            const float4 w = p0[(6 * blk + c) * step];
            x[c] = c2{make_float2(w.x, w.y), make_float2(w.z, w.w)};
        }
    }
    LYM_HD SlotF slot(int r) const { return SlotF{(float *)v, stride, lognp, r}; }
};

// One RHS r of a FP16 pair-layout batch, as a single half-spinor view.
struct SlotH {
    __half *hv;
    float *norm;
    int stride, lognp, r;
    static constexpr bool kPerComponent = false;  // a store needs the whole site (its norm)
    LYM_HD SlotH par(int) const { return *this; }
    LYM_D size_t base(int w, int h) const
    {
        return (((((size_t)w * stride + h) << lognp) + (r >> 1)) << 3) + (r & 1);
    }
    template <typename R> LYM_D void load(int h, cx<R> s[12]) const
    {
        const float n = norm[((size_t)h << (lognp + 1)) + r];
#pragma unroll
        for (int w = 0; w < 6; ++w) {
            const size_t b = base(w, h);
            s[2 * w] = cx<R>{(R)(__half2float(hv[b]) * n), (R)(__half2float(hv[b + 2]) * n)};
            s[2 * w + 1] = cx<R>{(R)(__half2float(hv[b + 4]) * n), (R)(__half2float(hv[b + 6]) * n)};
        }
    }
    template <typename R> LYM_D void store(int h, const cx<R> s[12]) const
    {
        float m = 0.f;
#pragma unroll
        for (int k = 0; k < 12; ++k) m = fmaxf(m, fmaxf(fabsf((float)s[k].re), fabsf((float)s[k].im)));
        const HalfScale sc(m);
        norm[((size_t)h << (lognp + 1)) + r] = m;
#pragma unroll
        for (int w = 0; w < 6; ++w) {
            const size_t b = base(w, h);
            hv[b] = __float2half_rn(sc((float)s[2 * w].re));
            hv[b + 2] = __float2half_rn(sc((float)s[2 * w].im));
            hv[b + 4] = __float2half_rn(sc((float)s[2 * w + 1].re));
            hv[b + 6] = __float2half_rn(sc((float)s[2 * w + 1].im));
        }
    }
};

struct BatchH {
    int4 *v;
    float2 *norm;
    int stride, lognp;
    LYM_D unsigned at(int w, int h, int q) const { return (((unsigned)w * stride + h) << lognp) + q; }
    LYM_D void load(int h, int q, c2 x[12]) const
    {
        const float2 n = __ldg(norm + ((unsigned)h << lognp) + q);
        const unsigned b = at(0, h, q), s = (unsigned)stride << lognp;
#pragma unroll
        for (int w = 0; w < 6; ++w) {
            int4 u = __ldg(v + b + w * s);
            const __half2 *hp = reinterpret_cast<const __half2 *>(&u);
            x[2 * w] = c2{mul2(__half22float2(hp[0]), n), mul2(__half22float2(hp[1]), n)};
            x[2 * w + 1] = c2{mul2(__half22float2(hp[2]), n), mul2(__half22float2(hp[3]), n)};
        }
    }
    LYM_D void load_cs(int h, int q, c2 x[12]) const { load(h, q, x); }
    LYM_D void store(int h, int q, const c2 x[12]) const
    {
        float ma = 0.f, mb = 0.f;
#pragma unroll
        for (int c = 0; c < 12; ++c) {
            ma = fmaxf(ma, fmaxf(fabsf(x[c].re.x), fabsf(x[c].im.x)));
            mb = fmaxf(mb, fmaxf(fabsf(x[c].re.y), fabsf(x[c].im.y)));
        }
        const HalfScale sa(ma), sb(mb);
        const float2 pre = make_float2(sa.pre, sb.pre), inv = make_float2(sa.inv, sb.inv);
        norm[((unsigned)h << lognp) + q] = make_float2(ma, mb);
        const unsigned b = at(0, h, q), s = (unsigned)stride << lognp;
#pragma unroll
        for (int w = 0; w < 6; ++w) {
            int4 u;
            __half2 *hp = reinterpret_cast<__half2 *>(&u);
            hp[0] = __float22half2_rn(mul2(mul2(x[2 * w].re, pre), inv));
            hp[1] = __float22half2_rn(mul2(mul2(x[2 * w].im, pre), inv));
            hp[2] = __float22half2_rn(mul2(mul2(x[2 * w + 1].re, pre), inv));
            hp[3] = __float22half2_rn(mul2(mul2(x[2 * w + 1].im, pre), inv));
            v[b + w * s] = u;
        }
    }
    LYM_D void get(int h, int q, int c, cx<double> &a, cx<double> &b) const
    {
        const float2 n = __ldg(norm + ((unsigned)h << lognp) + q);
        int4 u = __ldg(v + at(c >> 1, h, q));
        const __half2 *hp = reinterpret_cast<const __half2 *>(&u);
        const float2 re = mul2(__half22float2(hp[2 * (c & 1)]), n), im = mul2(__half22float2(hp[2 * (c & 1) + 1]), n);
        a = cx<double>{(double)re.x, (double)im.x};
        b = cx<double>{(double)re.y, (double)im.y};
    }
    LYM_D void load_d(int h, int q, cx<double> a[12], cx<double> b[12]) const
    {
        c2 x[12];
        load(h, q, x);
#pragma unroll
        for (int c = 0; c < 12; ++c) {
            a[c] = cx<double>{(double)x[c].re.x, (double)x[c].im.x};
            b[c] = cx<double>{(double)x[c].re.y, (double)x[c].im.y};
        }
    }
    LYM_D void store_d(int h, int q, const cx<double> a[12], const cx<double> b[12]) const
    {
        c2 x[12];
#pragma unroll
        for (int c = 0; c < 12; ++c)
            x[c] = c2{make_float2((float)a[c].re, (float)b[c].re), make_float2((float)a[c].im, (float)b[c].im)};
        store(h, q, x);
    }
    // the 6 words and the norm (word 6) through shared memory, as BatchF::stage / unstage
    LYM_D void stage(unsigned s0, unsigned sstep, int h, int q) const
    {
        const unsigned b = at(0, h, q), s = (unsigned)stride << lognp;
#pragma unroll
        for (int w = 0; w < 6; ++w) cp_async16(s0 + w * sstep, v + b + w * s);
        cp_async8(s0 + 6 * sstep, norm + ((unsigned)h << lognp) + q);
    }
    LYM_D void unstage(const float4 *p0, int step, c2 x[12]) const
    {
        const float4 nw = p0[6 * step];
        const float2 n = make_float2(nw.x, nw.y);
#pragma unroll
        for (int w = 0; w < 6; ++w) {
            const int4 u = *reinterpret_cast<const int4 *>(p0 + w * step);
            const __half2 *hp = reinterpret_cast<const __half2 *>(&u);
            x[2 * w] = c2{mul2(__half22float2(hp[0]), n), mul2(__half22float2(hp[1]), n)};
            x[2 * w + 1] = c2{mul2(__half22float2(hp[2]), n), mul2(__half22float2(hp[3]), n)};
        }
    }
    LYM_D void unstage_block(const float4 *p0, int step, int blk, c2 x[6]) const
    {
        const float4 nw = p0[6 * step];
        const float2 n = make_float2(nw.x, nw.y);
#pragma unroll
        for (int w = 0; w < 3; ++w) {
            const int4 u = *reinterpret_cast<const int4 *>(p0 + (3 * blk + w) * step);
            const __half2 *hp = reinterpret_cast<const __half2 *>(&u);
            x[2 * w] = c2{mul2(__half22float2(hp[0]), n), mul2(__half22float2(hp[1]), n)};
            x[2 * w + 1] = c2{mul2(__half22float2(hp[2]), n), mul2(__half22float2(hp[3]), n)};
        }
    }
    LYM_HD SlotH slot(int r) const { return SlotH{(__half *)v, (float *)norm, stride, lognp, r}; }
};

// ---------------------------------------------------------- links, clover --
struct LinkP {  // a link with every component duplicated into both lanes
    float2 ur[3][3], ui[3][3];
};

// Links and clover words are read by exactly one warp instruction per launch (all np
// lanes of the half-site at once), so they are loaded with the evict-first hint and
// leave L2 to the neighbour spinors, which are read eight times.
//
// GaugeC12P / GaugeR6P read the 12-real FP32 words of the single-RHS stencils (GaugeF12 /
// GaugeF6: rows 0 and 1, row 2 = s conj(row0 x row1), s = -1 where bit mu of the site's
// sign byte is set); GaugeF18P reads all 18 reals.  Either is expanded in registers into
// lane-duplicated components for the packed arithmetic.  Staged through shared memory, a
// 12-real link takes kStageWords slots: its 3 words and the aligned 32-bit word of the
// sign table that holds its sign byte.
LYM_D void cp_async4(unsigned saddr, const void *g)
{
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(saddr), "l"(g) : "memory");
}

struct GaugeC12P {  // SU(3)
    static constexpr bool kReal = false;
    static constexpr int kStageWords = 4;
    const float4 *u;       // [parity][mu][3][stride]
    const uint8_t *sign;   // [parity][stride]
    int stride;
    LYM_D static void expand(const float4 w0, const float4 w1, const float4 w2, unsigned neg, LinkP &L)
    {
        const float r[2][3] = {{w0.x, w0.z, w1.x}, {w1.z, w2.x, w2.z}};
        const float i[2][3] = {{w0.y, w0.w, w1.y}, {w1.w, w2.y, w2.w}};
#pragma unroll
        for (int a = 0; a < 2; ++a)
#pragma unroll
            for (int b = 0; b < 3; ++b) {
                L.ur[a][b] = make_float2(r[a][b], r[a][b]);
                L.ui[a][b] = make_float2(i[a][b], i[a][b]);
            }
        const float s = neg ? -1.f : 1.f;
#pragma unroll
        for (int j = 0; j < 3; ++j) {  // row 2 = s conj(r0_a r1_c - r0_c r1_a)
            const int a = (j + 1) % 3, c = (j + 2) % 3;
            const float vr = (r[0][a] * r[1][c] - i[0][a] * i[1][c]) - (r[0][c] * r[1][a] - i[0][c] * i[1][a]);
            const float vi = (r[0][a] * i[1][c] + i[0][a] * r[1][c]) - (r[0][c] * i[1][a] + i[0][c] * r[1][a]);
            L.ur[2][j] = make_float2(s * vr, s * vr);
            L.ui[2][j] = make_float2(-s * vi, -s * vi);
        }
    }
    LYM_D void load(int p, int mu, int h, LinkP &L) const
    {
        const float4 *b = u + ((unsigned)(p * 4 + mu) * 3 * stride + h);
        const float4 w0 = __ldcs(b), w1 = __ldcs(b + stride), w2 = __ldcs(b + 2 * stride);
        expand(w0, w1, w2, (__ldg(sign + (unsigned)p * stride + h) >> mu) & 1u, L);
    }
    // slot k of link (p, mu, h): words 0..2, then the sign word
    LYM_D void stage(int p, int mu, int k, int h, unsigned saddr) const
    {
        if (k < 3) cp_async16(saddr, u + ((unsigned)((p * 4 + mu) * 3 + k) * stride + h));
        else cp_async4(saddr, sign + (((unsigned)p * stride + h) & ~3u));
    }
    LYM_D void unstage(const float4 *w4, int mu, int h, LinkP &L) const
    {
        const unsigned word = *reinterpret_cast<const unsigned *>(w4 + 3);
        expand(w4[0], w4[1], w4[2], (word >> (8 * (h & 3) + mu)) & 1u, L);
    }
};

// SU(3) links in all 18 reals, entries row-major two per word (the boundary sign is part
// of the stored link): 5 words staged per link and no row to rebuild, against 3 words and a
// sign byte for GaugeC12P, whose rebuilt row costs every thread of the half-site about 50
// scalar instructions per link
struct GaugeF18P {
    static constexpr bool kReal = false;
    static constexpr int kStageWords = 5;
    const float4 *u;  // [parity][mu][5][stride]
    int stride;
    LYM_D static void expand(const float4 w0, const float4 w1, const float4 w2, const float4 w3, const float4 w4,
                             LinkP &L)
    {
        const float r[9] = {w0.x, w0.z, w1.x, w1.z, w2.x, w2.z, w3.x, w3.z, w4.x};
        const float i[9] = {w0.y, w0.w, w1.y, w1.w, w2.y, w2.w, w3.y, w3.w, w4.y};
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
            for (int b = 0; b < 3; ++b) {
                L.ur[a][b] = make_float2(r[3 * a + b], r[3 * a + b]);
                L.ui[a][b] = make_float2(i[3 * a + b], i[3 * a + b]);
            }
    }
    LYM_D void load(int p, int mu, int h, LinkP &L) const
    {
        const float4 *b = u + ((unsigned)(p * 4 + mu) * 5 * stride + h);
        expand(__ldcs(b), __ldcs(b + stride), __ldcs(b + 2 * stride), __ldcs(b + 3 * stride), __ldcs(b + 4 * stride), L);
    }
    LYM_D void stage(int p, int mu, int k, int h, unsigned saddr) const
    {
        cp_async16(saddr, u + ((unsigned)((p * 4 + mu) * 5 + k) * stride + h));
    }
    LYM_D void unstage(const float4 *w4, int, int, LinkP &L) const { expand(w4[0], w4[1], w4[2], w4[3], w4[4], L); }
};

struct GaugeR6P {  // real adjoint links: 3 float2 words (rows 0 and 1), row 2 = s (row0 x row1)
    static constexpr bool kReal = true;
    static constexpr int kStageWords = 4;
    const float2 *u;       // [parity][mu][3][stride]
    const uint8_t *sign;   // [parity][stride]
    int stride;
    LYM_D static void expand(const float2 w0, const float2 w1, const float2 w2, unsigned neg, LinkP &L)
    {
        const float r[2][3] = {{w0.x, w0.y, w1.x}, {w1.y, w2.x, w2.y}};
#pragma unroll
        for (int a = 0; a < 2; ++a)
#pragma unroll
            for (int b = 0; b < 3; ++b) L.ur[a][b] = make_float2(r[a][b], r[a][b]);
        const float s = neg ? -1.f : 1.f;
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            const int a = (j + 1) % 3, c = (j + 2) % 3;
            const float v = s * (r[0][a] * r[1][c] - r[0][c] * r[1][a]);
            L.ur[2][j] = make_float2(v, v);
        }
    }
    LYM_D void load(int p, int mu, int h, LinkP &L) const
    {
        const float2 *b = u + ((unsigned)(p * 4 + mu) * 3 * stride + h);
        const float2 w0 = __ldcs(b), w1 = __ldcs(b + stride), w2 = __ldcs(b + 2 * stride);
        expand(w0, w1, w2, (__ldg(sign + (unsigned)p * stride + h) >> mu) & 1u, L);
    }
    LYM_D void stage(int p, int mu, int k, int h, unsigned saddr) const
    {
        if (k < 3) cp_async8(saddr, u + ((unsigned)((p * 4 + mu) * 3 + k) * stride + h));
        else cp_async4(saddr, sign + (((unsigned)p * stride + h) & ~3u));
    }
    LYM_D void unstage(const float4 *w4, int mu, int h, LinkP &L) const
    {
        const unsigned word = *reinterpret_cast<const unsigned *>(w4 + 3);
        expand(make_float2(w4[0].x, w4[0].y), make_float2(w4[1].x, w4[1].y), make_float2(w4[2].x, w4[2].y),
               (word >> (8 * (h & 3) + mu)) & 1u, L);
    }
};

// w = U h.  Re w_i = sum_j Ur_ij Re h_j - sum_j Ui_ij Im h_j: the subtracted sum is
// accumulated on its own and taken off once per row, so no negated operand is needed.
template <bool REAL> LYM_D void mul_u2(const LinkP &L, const c2 h[3], c2 w[3])
{
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        float2 re = mul2(L.ur[i][0], h[0].re), im = mul2(L.ur[i][0], h[0].im);
#pragma unroll
        for (int j = 1; j < 3; ++j) {
            re = fma2(L.ur[i][j], h[j].re, re);
            im = fma2(L.ur[i][j], h[j].im, im);
        }
        if (!REAL) {
            float2 t = mul2(L.ui[i][0], h[0].im);
#pragma unroll
            for (int j = 1; j < 3; ++j) t = fma2(L.ui[i][j], h[j].im, t);
#pragma unroll
            for (int j = 0; j < 3; ++j) im = fma2(L.ui[i][j], h[j].re, im);
            re = sub2(re, t);
        }
        w[i] = c2{re, im};
    }
}

// w = U^+ h.  Im w_i = sum_j Ur_ji Im h_j - sum_j Ui_ji Re h_j.
template <bool REAL> LYM_D void mul_ud2(const LinkP &L, const c2 h[3], c2 w[3])
{
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        float2 re = mul2(L.ur[0][i], h[0].re), im = mul2(L.ur[0][i], h[0].im);
#pragma unroll
        for (int j = 1; j < 3; ++j) {
            re = fma2(L.ur[j][i], h[j].re, re);
            im = fma2(L.ur[j][i], h[j].im, im);
        }
        if (!REAL) {
            float2 t = mul2(L.ui[0][i], h[0].re);
#pragma unroll
            for (int j = 1; j < 3; ++j) t = fma2(L.ui[j][i], h[j].re, t);
#pragma unroll
            for (int j = 0; j < 3; ++j) re = fma2(L.ui[j][i], h[j].im, re);
            im = sub2(im, t);
        }
        w[i] = c2{re, im};
    }
}

// Clover words of one half-site for a pair: word k (0..8) of block blk as four lane
// pairs.  From shared memory when the whole batch shares one operator (each value is
// duplicated into both lanes), else from each lane's own clover term in HBM.
struct CloverWordsSmem {
    const float4 *w0, *w1;  // the 9 words of block 0 and of block 1
    LYM_D void get(int blk, int k, float2 v[4]) const
    {
        const float4 x = (blk ? w1 : w0)[k];
        v[0] = make_float2(x.x, x.x);
        v[1] = make_float2(x.y, x.y);
        v[2] = make_float2(x.z, x.z);
        v[3] = make_float2(x.w, x.w);
    }
};
struct CloverWordsGlobal {
    const float4 *ta, *tb;
    unsigned base;  // (p * 2 * 9) * stride + h
    int stride;
    bool same;
    LYM_D void get(int blk, int k, float2 v[4]) const
    {
        const unsigned o = base + (unsigned)(blk * 9 + k) * stride;
        const float4 wa = __ldcs(ta + o);
        const float4 wb = same ? wa : __ldcs(tb + o);
        v[0] = make_float2(wa.x, wb.x);
        v[1] = make_float2(wa.y, wb.y);
        v[2] = make_float2(wa.z, wb.z);
        v[3] = make_float2(wa.w, wb.w);
    }
};

LYM_HD constexpr int tri_row(int t) { return t < 1 ? 1 : t < 3 ? 2 : t < 6 ? 3 : t < 10 ? 4 : 5; }

// out = SIGN (add + A x) for one Hermitian 6x6 block A of the FP32 clover term (packed as
// in CloverF: 6 real diagonal entries, then the 15 entries below the diagonal, row-major),
// for the two RHS of a pair.  With HAS_ADD, out holds SIGN * add on entry (the block is
// accumulated in place); without it out is written.  The words are read one at a time in
// storage order; products entering with the other sign are summed apart (nre, nim) and
// subtracted once per row, so no negated operand is formed.
template <int SIGN, bool HAS_ADD, class CW> LYM_D void clover_block_apply(const CW &cw, int blk, const c2 x[6], c2 out[6])
{
    // the products that enter with a minus sign take a negated word (one negation per word,
    // shared by its uses), so no separate accumulators are held
#pragma unroll
    for (int k = 0; k < 9; ++k) {
        float2 w[4];
        cw.get(blk, k, w);
        if (SIGN < 0)
#pragma unroll
            for (int l = 0; l < 4; ++l) w[l] = make_float2(-w[l].x, -w[l].y);
#pragma unroll
        for (int l = 0; l < 4; ++l) {
            const int e = 4 * k + l;
            if (e < 6) {  // diagonal entry d_e (the first words: every row starts here)
                out[e].re = HAS_ADD ? fma2(w[l], x[e].re, out[e].re) : mul2(w[l], x[e].re);
                out[e].im = HAS_ADD ? fma2(w[l], x[e].im, out[e].im) : mul2(w[l], x[e].im);
            } else if (((e - 6) & 1) == 0) {  // entry t = (i, j), i > j: (re, im) = w[l], w[l + 1]
                const int t = (e - 6) / 2, i = tri_row(t), j = t - i * (i - 1) / 2;
                const float2 are = w[l], aim = w[l + 1], naim = make_float2(-aim.x, -aim.y);
                // y_i += a x_j
                out[i].re = fma2(are, x[j].re, out[i].re);
                out[i].re = fma2(naim, x[j].im, out[i].re);
                out[i].im = fma2(are, x[j].im, out[i].im);
                out[i].im = fma2(aim, x[j].re, out[i].im);
                // y_j += conj(a) x_i
                out[j].re = fma2(are, x[i].re, out[j].re);
                out[j].re = fma2(aim, x[i].im, out[j].re);
                out[j].im = fma2(are, x[i].im, out[j].im);
                out[j].im = fma2(naim, x[i].re, out[j].im);
            }
        }
    }
}

// ---------------------------------------------------------- batch stencil --
// One term of H x for the pair: DIR 0 adds U_mu(s) (1 - g_mu) x(s + mu), DIR 1 adds
// U_mu(s - mu)^+ (1 + g_mu) x(s - mu), through the half-spinor projections of the
// chiral basis (see lym_dslash.cuh).
template <bool REAL, int MU, int DIR> LYM_D void accumulate_dir(const c2 x[12], const LinkP &L, c2 acc[12])
{
#pragma unroll
    for (int k = 0; k < 2; ++k) {
        const int code = proj_code(MU, k), pk = proj_partner(MU, k);
        c2 hv[3], w[3];
#pragma unroll
        for (int m = 0; m < 3; ++m)
            hv[m] = DIR == 0 ? add_code<-1>(x[3 * k + m], code, x[3 * pk + m])
                             : add_code<+1>(x[3 * k + m], code, x[3 * pk + m]);
        if (DIR == 0) mul_u2<REAL>(L, hv, w);
        else mul_ud2<REAL>(L, hv, w);
#pragma unroll
        for (int m = 0; m < 3; ++m) {
            acc[3 * k + m] = c2{add2(acc[3 * k + m].re, w[m].re), add2(acc[3 * k + m].im, w[m].im)};
            acc[3 * pk + m] = DIR == 0 ? add_code<-1>(acc[3 * pk + m], conj_code(code), w[m])
                                       : add_code<+1>(acc[3 * pk + m], conj_code(code), w[m]);
        }
    }
}

template <bool REAL, int MU, class SB, class GaugeT>
LYM_D void hopping_mu(const int nf[4], const int nbk[4], const SB &in, const GaugeT &U, int p, int h, int q,
                      c2 acc[12])
{
    {
        c2 x[12];
        in.load(nf[MU], q, x);
        LinkP L;
        U.load(p, MU, h, L);
        accumulate_dir<REAL, MU, 0>(x, L, acc);
    }
    {
        c2 x[12];
        in.load(nbk[MU], q, x);
        LinkP L;
        U.load(1 - p, MU, nbk[MU], L);
        accumulate_dir<REAL, MU, 1>(x, L, acc);
    }
}

// H x at half-site h of output parity p for the pair q; nf / nbk: the forward and
// backward neighbour half-sites, read from the table before the first spinor load.
template <bool REAL, class SB, class GaugeT>
LYM_D void hopping_pair(const int nf[4], const int nbk[4], const SB &in, const GaugeT &U, int p, int h, int q,
                        c2 acc[12])
{
#pragma unroll
    for (int k = 0; k < 12; ++k) acc[k] = c2{make_float2(0.f, 0.f), make_float2(0.f, 0.f)};
    hopping_mu<REAL, 0>(nf, nbk, in, U, p, h, q, acc);
    hopping_mu<REAL, 1>(nf, nbk, in, U, p, h, q, acc);
    hopping_mu<REAL, 2>(nf, nbk, in, U, p, h, q, acc);
    hopping_mu<REAL, 3>(nf, nbk, in, U, p, h, q, acc);
}

// threads per block of the shared-memory staged stencil (dslash_batch_staged_kernel)
constexpr int kStagedThreads = 128;

// Work item -> half-site and its 8 neighbours by arithmetic, for the traversal in (y, z)
// columns of by x bz (the order of order_table_kernel; h order is the column Ly x Lz):
// w = th + lth (zi + bz (yi + by (x + Lx (zb + nzb yb)))), th = t / 2, lth = Lt / 2.
// Divisions are multiply-high by m = ceil(2^32 / d), exact for w < 2^24 and d <= 256
// (the host checks both before it enables the walk).
struct ColumnWalk {
    int on;                           // 0: use the order and neighbour tables
    int L[4], lth, by, bz, nzb;
    unsigned m_lth, m_bz, m_by, m_lx, m_nzb;  // 0 for a divisor of 1
};

LYM_D unsigned walk_div(unsigned n, unsigned m) { return m ? __umulhi(n, m) : n; }

// h and the neighbour half-sites nf (+mu) and nbk (-mu) of work item w at output parity p
LYM_D int walk_site(const ColumnWalk &cw, int p, unsigned w, int nf[4], int nbk[4])
{
    unsigned u = w, q;
    q = walk_div(u, cw.m_lth);
    const int th = (int)(u - q * cw.lth);
    u = q;
    q = walk_div(u, cw.m_bz);
    const int zi = (int)(u - q * cw.bz);
    u = q;
    q = walk_div(u, cw.m_by);
    const int yi = (int)(u - q * cw.by);
    u = q;
    q = walk_div(u, cw.m_lx);
    const int x = (int)(u - q * cw.L[0]);
    u = q;
    q = walk_div(u, cw.m_nzb);
    const int zb = (int)(u - q * cw.nzb), yb = (int)q;
    const int y = yb * cw.by + yi, z = zb * cw.bz + zi;
    const int t = 2 * th + ((p + x + y + z) & 1);
    const int sx = cw.lth * cw.L[2] * cw.L[1], sy = cw.lth * cw.L[2], sz = cw.lth;
    const int h = th + sz * z + sy * y + sx * x;
    nf[0] = h + (x + 1 == cw.L[0] ? -x * sx : sx);
    nbk[0] = h + (x == 0 ? (cw.L[0] - 1) * sx : -sx);
    nf[1] = h + (y + 1 == cw.L[1] ? -y * sy : sy);
    nbk[1] = h + (y == 0 ? (cw.L[1] - 1) * sy : -sy);
    nf[2] = h + (z + 1 == cw.L[2] ? -z * sz : sz);
    nbk[2] = h + (z == 0 ? (cw.L[2] - 1) * sz : -sz);
    const int base = h - th;
    nf[3] = base + ((t + 1 == cw.L[3] ? 0 : t + 1) >> 1);
    nbk[3] = base + ((t == 0 ? cw.L[3] - 1 : t - 1) >> 1);
    return h;
}

template <class SB, class GaugeT> struct DslashBatchArg {
    Geom g;
    SB in, out, y;
    GaugeT U;
    int parity, gamma5, has_clover, lognp;
    float a, b;
    NbrTable nbr;        // precomputed neighbour half-site indices
    const int *order;    // work item -> half-site ([stride], both parities) or nullptr
    const int *skip_if;  // skip the launch when *skip_if != 0
    const int *active;   // per-RHS mask (nullptr: all active)
    // per-RHS operator: slots of one batch share the gauge field but may carry different
    // kappa, hence different b (nullptr: the shared b) and clover terms (FP32 bases)
    const double *b_slot;
    const void *const *clover_slot;
    const int *uniform;  // device flag: every slot on one operator (nullptr: not known)
    // EPI_XPAY_RES: the BiCGStab residual s = r - alpha out of every active RHS (an inactive
    // lane copies r), written next to out
    BatchF res_r;
    SB res_s;
    const double2 *res_alpha;
    // EPI_XPAY_OMEGA: rhat and the per-block partial sums [block][nb][7]
    BatchF om_rhat;
    double *om_partials;
    ColumnWalk walk;  // the staged kernel's indices without tables (walk.on)
    int *err;         // bulk-copy variant: set to 1 when a copy wait gave up
};

struct NoWait {
    LYM_D void operator()() const {}
};

// The epilogue on H x (acc) for the pair q at half-site h, written to out.  ysrc(blk, y6)
// gives the 6 same-parity input components of block blk (EPI_XPAY); cw the clover words.
// before_blk1() runs before anything of spin block 1, the clover words of that block or the
// fused epilogue's own-site operand (r_smem) is read (the staged kernel waits there for the
// copies it issued after the last direction).
template <int EPI, class SB, class GaugeT, class YSrc, class CW, class Wait = NoWait>
LYM_D void batch_epilogue(const DslashBatchArg<SB, GaugeT> &arg, int h, int q, bool act_a, bool act_b, c2 acc[12],
                          const YSrc &ysrc, const CW &cw, const float4 *r_smem = nullptr,
                          const Wait &before_blk1 = Wait{})
{
    const int ra = 2 * q, rb = 2 * q + 1;
    if (EPI == EPI_SCALE || EPI == EPI_CLOVINV) {
        const float2 a = make_float2(arg.a, arg.a);
#pragma unroll
        for (int k = 0; k < 12; ++k) acc[k] = c2{mul2(a, acc[k].re), mul2(a, acc[k].im)};
        if (EPI == EPI_CLOVINV && arg.has_clover) {
#pragma unroll
            for (int blk = 0; blk < 2; ++blk) {
                if (blk == 1) before_blk1();
                c2 res[6];
                clover_block_apply<+1, false>(cw, blk, acc + 6 * blk, res);
#pragma unroll
                for (int k = 0; k < 6; ++k) acc[6 * blk + k] = res[k];
            }
        }
    } else {
        float ba = arg.b, bb = arg.b;
        if (arg.b_slot) {
            ba = (float)arg.b_slot[act_a ? ra : rb];
            bb = (float)arg.b_slot[act_b ? rb : ra];
        }
        const float2 b = make_float2(ba, bb), nb = make_float2(-ba, -bb);
#pragma unroll
        for (int blk = 0; blk < 2; ++blk) {
            if (blk == 1) before_blk1();
            c2 y6[6];
            ysrc(blk, y6);
            c2 *o = acc + 6 * blk;
            if (blk == 1 && arg.gamma5) {  // lower spins: -(T y + b H x)
#pragma unroll
                for (int k = 0; k < 6; ++k) o[k] = c2{mul2(nb, o[k].re), mul2(nb, o[k].im)};
                if (arg.has_clover) {
                    clover_block_apply<-1, true>(cw, blk, y6, o);
                } else {
#pragma unroll
                    for (int k = 0; k < 6; ++k) o[k] = c2{sub2(o[k].re, y6[k].re), sub2(o[k].im, y6[k].im)};
                }
            } else {
#pragma unroll
                for (int k = 0; k < 6; ++k) o[k] = c2{mul2(b, o[k].re), mul2(b, o[k].im)};
                if (arg.has_clover) {
                    clover_block_apply<+1, true>(cw, blk, y6, o);
                } else {
#pragma unroll
                    for (int k = 0; k < 6; ++k) o[k] = c2{add2(o[k].re, y6[k].re), add2(o[k].im, y6[k].im)};
                }
            }
        }
    }
    arg.out.store(h, q, acc);
    if constexpr (EPI == EPI_XPAY_RES) {
        before_blk1();
        c2 r[12];  // r from this thread's shared-memory slots (staged kernel) or from memory
        if (r_smem) arg.res_r.unstage(r_smem, kStagedThreads, r);
        else arg.res_r.load(h, q, r);
        const double2 aa = act_a ? arg.res_alpha[ra] : make_double2(0.0, 0.0);
        const double2 ab = act_b ? arg.res_alpha[rb] : make_double2(0.0, 0.0);
        const float2 are = make_float2((float)aa.x, (float)ab.x), aim = make_float2((float)aa.y, (float)ab.y);
#pragma unroll
        for (int k = 0; k < 12; ++k) {
            // s = r - alpha v:  re -= are v.re - aim v.im,  im -= are v.im + aim v.re
            const float2 sre = fma2(aim, acc[k].im, sub2(r[k].re, mul2(are, acc[k].re)));
            const float2 sim = sub2(sub2(r[k].im, mul2(are, acc[k].im)), mul2(aim, acc[k].re));
            r[k] = c2{sre, sim};
        }
        arg.res_s.store(h, q, r);
    }
}

template <int EPI, class SB, class GaugeT>
LYM_D CloverWordsGlobal clover_global(const DslashBatchArg<SB, GaugeT> &arg, int h, int q, bool act_a, bool act_b)
{
    CloverWordsGlobal cw{nullptr, nullptr, (unsigned)arg.parity * 18 * arg.g.stride + h, arg.g.stride, true};
    if (EPI != EPI_SCALE && arg.has_clover) {  // an inactive lane borrows its partner's operator
        cw.ta = (const float4 *)arg.clover_slot[act_a ? 2 * q : 2 * q + 1];
        cw.tb = (const float4 *)arg.clover_slot[act_b ? 2 * q + 1 : 2 * q];
        cw.same = cw.ta == cw.tb;
    }
    return cw;
}

// out_r = a H in_r (EPI_SCALE), Tinv_r (a H in_r) (EPI_CLOVINV) or
// G5^g (T_r y_r + b_r H in_r) (EPI_XPAY), for both RHS of every pair with an active RHS
template <int EPI, int MINB, class SB, class GaugeT>
__global__ void __launch_bounds__(128, MINB) dslash_batch_kernel(const DslashBatchArg<SB, GaugeT> arg)
{
    if (arg.skip_if && *arg.skip_if) return;
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    const int wi = tid >> arg.lognp, q = tid & ((1 << arg.lognp) - 1);
    if (wi >= arg.g.Vh) return;
    bool act_a = true, act_b = true;
    if (arg.active) {
        act_a = arg.active[2 * q] != 0;
        act_b = arg.active[2 * q + 1] != 0;
        if (!act_a && !act_b) return;
    }
    int h, nf[4], nbk[4];
    if (arg.walk.on) {
        h = walk_site(arg.walk, arg.parity, (unsigned)wi, nf, nbk);
    } else {
        h = arg.order ? __ldg(arg.order + wi) : wi;
#pragma unroll
        for (int mu = 0; mu < 4; ++mu) {
            nf[mu] = arg.nbr.get(arg.parity, mu, 0, h);
            nbk[mu] = arg.nbr.get(arg.parity, mu, 1, h);
        }
    }
    c2 acc[12];
    hopping_pair<GaugeT::kReal>(nf, nbk, arg.in, arg.U, arg.parity, h, q, acc);
    const CloverWordsGlobal cw = clover_global<EPI>(arg, h, q, act_a, act_b);
    if (EPI == EPI_XPAY || EPI == EPI_XPAY_RES) {
        c2 yv[12];
        arg.y.load_cs(h, q, yv);
        batch_epilogue<EPI>(arg, h, q, act_a, act_b, acc, [&](int blk, c2 y6[6]) {
#pragma unroll
            for (int k = 0; k < 6; ++k) y6[k] = yv[6 * blk + k];
        }, cw);
    } else {
        batch_epilogue<EPI>(arg, h, q, act_a, act_b, acc, [](int, c2 *) {}, cw);
    }
}

// ------------------------------------------------------ staged batch stencil --
// The same stencil with the neighbour spinors and links of direction d + 1 copied into
// shared memory (cp.async) while direction d is computed, so the loads of the next
// term overlap the arithmetic of this one without holding registers.  Shared memory
// per block of 128 threads: two buffers of 12 words per thread (the thread's own
// spinor words) and two buffers of 9 words per half-site (a link's kStageWords words, or
// the clover words of a batch on one operator); the np threads of a half-site copy its
// link words between them and meet at __syncwarp before reading.
LYM_HD int staged_smem_bytes(int lognp)
{
    // spinor buffers, link / clover slots, then one mbarrier per (buffer, half-site) of the
    // bulk-copy variant
    return (2 * 12 * kStagedThreads + 2 * (kStagedThreads >> lognp) * 9) * 16 + 2 * (kStagedThreads >> lognp) * 8;
}

// BULK: the neighbour spinor words of a direction arrive by bulk copies, one per component
// of the half-site (16 np contiguous bytes in global and in shared memory), completing on the
// half-site's mbarrier of that buffer (FP32 batches).  When a wait of any lane of the warp
// gives up, the warp issues no further bulk copies, raises the error word and, before it
// leaves, waits once more (bounded) for the copies it has in flight.
template <bool STAGE_Y, bool BULK, class SB, class GaugeT> struct StagedHop {
    const DslashBatchArg<SB, GaugeT> &arg;
    float4 *smem;
    int h, q, np, site, lane_in;
    int nf[4], nbk[4];
    bool live;
    unsigned vmask;
    bool clov_smem;       // the batch shares one operator: its clover words go through shared memory
    const float4 *clov;   // that operator's clover term
    int stalled = -1;     // BULK: the direction whose wait gave up (-1: none)

    // the 9 words of clover block blk of this half-site into link buffer blk
    LYM_D void stage_clover(int blk) const
    {
        const unsigned base = ((unsigned)(arg.parity * 2 + blk) * 9) * arg.g.stride + h;
        float4 *L = sl(blk);
        for (int k = lane_in; k < 9; k += np) cp_async16(smem_u32(L + k), clov + base + k * arg.g.stride);
    }

    LYM_D float4 *sx(int buf) const { return smem + buf * 12 * kStagedThreads + threadIdx.x; }
    LYM_D unsigned mbar(int buf) const
    {
        const float4 *after = smem + 2 * 12 * kStagedThreads + 2 * (kStagedThreads / np) * 9;
        return smem_u32(after) + (unsigned)(buf * (kStagedThreads / np) + site) * 8u;
    }
    LYM_D void init_bulk() const
    {
        if (lane_in == 0) {
            mbar_init(mbar(0));
            mbar_init(mbar(1));
            mbar_init_fence();
        }
        __syncwarp(vmask);
    }
    LYM_D float4 *sl(int buf) const
    {
        return smem + 2 * 12 * kStagedThreads + (buf * (kStagedThreads / np) + site) * 9;
    }
    template <int D> LYM_D void issue() const
    {
        constexpr int MU = D / 2, DIR = D % 2;
        const int n = DIR == 0 ? nf[MU] : nbk[MU];
        if constexpr (BULK) {
            if (stalled >= 0) return;  // nothing new after a wait gave up (the error word is set)
            const unsigned bytes = 16u * np, mb = mbar(D & 1);
            const unsigned dst0 = smem_u32(smem + (D & 1) * 12 * kStagedThreads + site * np);
            if (lane_in == 0) mbar_expect(mb, 12u * bytes);
            fence_proxy_async();
            for (int c = lane_in; c < 12; c += np)
                bulk_copy(dst0 + (unsigned)c * kStagedThreads * 16u, arg.in.v + arg.in.at(c, n, 0), bytes, mb);
        } else {
            if (live) arg.in.stage(smem_u32(sx(D & 1)), kStagedThreads * 16, n, q);
        }
        const int lp = DIR == 0 ? arg.parity : 1 - arg.parity, lh = DIR == 0 ? h : n;
        float4 *L = sl(D & 1);
        for (int k = lane_in; k < GaugeT::kStageWords; k += np) arg.U.stage(lp, MU, k, lh, smem_u32(L + k));
    }
    template <int D> LYM_D void step(c2 acc[12])
    {
        if constexpr (D < 7) {
            issue<D + 1>();
        } else {
            if (STAGE_Y && live) arg.y.stage(smem_u32(sx(0)), kStagedThreads * 16, h, q);
            if (clov_smem) stage_clover(0);
        }
        cp_async_commit();
        cp_async_wait<1>();  // the copies of direction D (this thread's)
        if constexpr (BULK) {  // its spinor words
            if (stalled < 0 && __any_sync(vmask, !mbar_wait(mbar(D & 1), (D >> 1) & 1))) {
                stalled = D;
                if (lane_in == 0) atomicOr(arg.err, 1);
            }
        }
        __syncwarp(vmask);   // ... and those of the other lanes of the half-site
        if (live) {
            c2 x[12];
            arg.in.unstage(sx(D & 1), kStagedThreads, x);
            LinkP L;
            arg.U.unstage(sl(D & 1), D / 2, D % 2 == 0 ? h : nbk[D / 2], L);
            accumulate_dir<GaugeT::kReal, D / 2, D % 2>(x, L, acc);
        }
        __syncwarp(vmask);  // every lane is done with buffer D & 1 before it is refilled
    }
    // BULK, after a wait gave up at direction d: the copies of d and of d + 1 (issued before
    // that wait) may still be in flight; wait for them, bounded, before the block leaves
    LYM_D void drain() const
    {
        if (stalled < 0) return;
        mbar_wait(mbar(stalled & 1), (stalled >> 1) & 1);
        if (stalled < 7) mbar_wait(mbar((stalled + 1) & 1), ((stalled + 1) >> 1) & 1);
    }
};

// EPI_XPAY_OMEGA: the sums of one thread's pair are reduced over the block in a fixed order
// (warp shuffles, then the four warps in shared memory) and written as the block's partial
// sums [block][nb][7]; every thread of the block takes part.
template <class SB, class GaugeT>
LYM_D void omega_block_reduce(const DslashBatchArg<SB, GaugeT> &arg, float4 *smem, double v[14])
{
    __syncthreads();  // every thread is done with the staging buffers
    double *sm = reinterpret_cast<double *>(smem);  // [4 warps][kMaxBatch][7]
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int np = 1 << arg.lognp, nb = 2 * np;
#pragma unroll
    for (int k = 0; k < 14; ++k)
        for (int o = 16; o >= np; o >>= 1) v[k] += __shfl_down_sync(0xffffffffu, v[k], o);
    if (lane < np) {
#pragma unroll
        for (int j = 0; j < 7; ++j) {
            sm[(warp * kMaxBatch + 2 * lane) * 7 + j] = v[j];
            sm[(warp * kMaxBatch + 2 * lane + 1) * 7 + j] = v[7 + j];
        }
    }
    __syncthreads();
    if ((int)threadIdx.x < nb) {
        for (int j = 0; j < 7; ++j) {
            double t = 0.0;
            for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += sm[(w * kMaxBatch + threadIdx.x) * 7 + j];
            arg.om_partials[((size_t)blockIdx.x * nb + threadIdx.x) * 7 + j] = t;
        }
    }
}

template <int EPI, int MINB, bool BULK, class SB, class GaugeT>
__global__ void __launch_bounds__(kStagedThreads, MINB)
    dslash_batch_staged_kernel(const DslashBatchArg<SB, GaugeT> arg)
{
    static_assert(!BULK || std::is_same<SB, BatchF>::value, "bulk copies stage FP32 batches");
    constexpr bool B = BULK;
    extern __shared__ float4 stage_smem[];
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    const int wi = tid >> arg.lognp, q = tid & ((1 << arg.lognp) - 1);
    const bool valid = wi < arg.g.Vh;  // equal for all lanes of a half-site
    constexpr bool RED = EPI == EPI_XPAY_OMEGA;
    // the flags of the launch and of this pair, loaded together: one memory latency before
    // the first copy is issued (the omega variant reads the pair's flags later: its
    // registers are taken by the sums)
    const int skip = arg.skip_if ? *arg.skip_if : 0;
    const bool uniform = !RED && EPI != EPI_SCALE && arg.has_clover && arg.uniform && *arg.uniform;
    int flag_a = 1, flag_b = 1;
    if (!RED && arg.active && valid) {
        flag_a = arg.active[2 * q];
        flag_b = arg.active[2 * q + 1];
    }
    if (skip) return;
    double red[RED ? 14 : 1];  // set by work() when it returns true
    const unsigned vmask = __ballot_sync(0xffffffffu, valid);
    auto work = [&]() -> bool {
        if (!valid) return false;
        if (RED && arg.active) {
            flag_a = arg.active[2 * q];
            flag_b = arg.active[2 * q + 1];
        }
        const bool act_a = flag_a != 0, act_b = flag_b != 0;
        const int np = 1 << arg.lognp;
        StagedHop<EPI == EPI_XPAY || EPI == EPI_XPAY_RES || EPI == EPI_XPAY_OMEGA, B, SB, GaugeT> s{
            arg, stage_smem, 0, q, np, (int)threadIdx.x >> arg.lognp, (int)threadIdx.x & (np - 1)};
        if (arg.walk.on) {
            s.h = walk_site(arg.walk, arg.parity, (unsigned)wi, s.nf, s.nbk);
        } else {
            s.h = arg.order ? __ldg(arg.order + wi) : wi;
#pragma unroll
            for (int mu = 0; mu < 4; ++mu) {
                s.nf[mu] = arg.nbr.get(arg.parity, mu, 0, s.h);
                s.nbk[mu] = arg.nbr.get(arg.parity, mu, 1, s.h);
            }
        }
        s.live = act_a || act_b;  // idle pairs still copy their share of the link words
        s.vmask = vmask;
        s.clov_smem = RED ? arg.has_clover && arg.uniform && *arg.uniform : uniform;
        s.clov = s.clov_smem ? (const float4 *)arg.clover_slot[0] : nullptr;
        c2 acc[12];
#pragma unroll
        for (int k = 0; k < 12; ++k) acc[k] = c2{make_float2(0.f, 0.f), make_float2(0.f, 0.f)};
        if constexpr (B) s.init_bulk();
        s.template issue<0>();
        cp_async_commit();
        s.template step<0>(acc);
        s.template step<1>(acc);
        s.template step<2>(acc);
        s.template step<3>(acc);
        s.template step<4>(acc);
        s.template step<5>(acc);
        s.template step<6>(acc);
        s.template step<7>(acc);
        if (s.clov_smem) s.stage_clover(1);  // link buffer 1 is free after the last direction
        // the own-site operand of a fused epilogue (r, rhat) into this thread's slots of
        // spinor buffer 1, free after the last direction as well
        if constexpr (EPI == EPI_XPAY_RES)
            if (s.live) arg.res_r.stage(smem_u32(s.sx(1)), kStagedThreads * 16, s.h, q);
        if constexpr (RED)
            if (s.live) arg.om_rhat.stage(smem_u32(s.sx(1)), kStagedThreads * 16, s.h, q);
        cp_async_commit();
        // the copies of step 7 (y, clover block 0) now; those just issued (clover block 1,
        // r or rhat) before the epilogue first reads them, so that their latency overlaps
        // block 0 of the epilogue.  Every lane of the half-site meets both warp barriers
        // (each waits for its own copies, which its neighbours read), a thread without an
        // active right-hand side before it leaves.
        cp_async_wait<1>();
        if constexpr (B) s.drain();
        __syncwarp(vmask);
        if (!s.live) {
            cp_async_wait<0>();
            __syncwarp(vmask);
            return false;
        }
        bool waited = false;
        auto wait_rest = [&]() {
            if (!waited) {
                cp_async_wait<0>();
                __syncwarp(vmask);
                waited = true;
            }
        };
        auto ysrc = [&](int blk, c2 y6[6]) { arg.y.unstage_block(s.sx(0), kStagedThreads, blk, y6); };
        if (s.clov_smem) {
            batch_epilogue<EPI>(arg, s.h, q, act_a, act_b, acc, ysrc, CloverWordsSmem{s.sl(0), s.sl(1)}, s.sx(1),
                                wait_rest);
        } else {
            batch_epilogue<EPI>(arg, s.h, q, act_a, act_b, acc, ysrc, clover_global<EPI>(arg, s.h, q, act_a, act_b),
                                s.sx(1), wait_rest);
        }
        wait_rest();
        if constexpr (RED) {
            // the omega sums of the two lanes: <t, s>, |t|^2, <rhat, s>, <rhat, t> (t = out,
            // s = y), over the 12 components of this half-site in packed FP32 (one lane per
            // RHS, a fixed order), then FP64 from the per-thread totals on: the block and
            // grid reductions add 2^22 and more such totals, each of 12 products
            const float2 zero = make_float2(0.f, 0.f);
            float2 P[7];
#pragma unroll
            for (int k = 0; k < 7; ++k) P[k] = zero;
#pragma unroll
            for (int blk = 0; blk < 2; ++blk) {
                c2 y6[6], r6[6];
                ysrc(blk, y6);
                arg.om_rhat.unstage_block(s.sx(1), kStagedThreads, blk, r6);
#pragma unroll
                for (int k = 0; k < 6; ++k) {
                    const c2 t = acc[6 * blk + k], sv = y6[k], rh = r6[k];
                    const float2 nti = sub2(zero, t.im), nri = sub2(zero, rh.im);
                    P[0] = fma2(t.im, sv.im, fma2(t.re, sv.re, P[0]));   // Re <t, s>
                    P[1] = fma2(nti, sv.re, fma2(t.re, sv.im, P[1]));    // Im <t, s>
                    P[2] = fma2(t.im, t.im, fma2(t.re, t.re, P[2]));     // |t|^2
                    P[3] = fma2(rh.im, sv.im, fma2(rh.re, sv.re, P[3])); // Re <rhat, s>
                    P[4] = fma2(nri, sv.re, fma2(rh.re, sv.im, P[4]));   // Im <rhat, s>
                    P[5] = fma2(rh.im, t.im, fma2(rh.re, t.re, P[5]));   // Re <rhat, t>
                    P[6] = fma2(nri, t.re, fma2(rh.re, t.im, P[6]));     // Im <rhat, t>
                }
            }
            // an idle lane's sums are dropped (its words may hold anything)
#pragma unroll
            for (int k = 0; k < 7; ++k) {
                red[k] = act_a ? (double)P[k].x : 0.0;
                red[7 + k] = act_b ? (double)P[k].y : 0.0;
            }
        }
        return true;
    };
    const bool summed = work();
    if constexpr (RED) {
        if (!summed)
#pragma unroll
            for (int k = 0; k < 14; ++k) red[k] = 0.0;
        omega_block_reduce(arg, stage_smem, red);
    }
}

// --------------------------------------------------- batch site kernels ----
// Like site_kernel, over (h, pair) items with the pair index fastest; each thread keeps
// one pair (the grid stride is a multiple of np), its FP64 partial sums are per RHS,
// acc[lane * NRED + k], and the last block runs Op::finalize(r, totals) for every r in
// parallel (thread r), then Op::finalize_all().
template <class Op>
__global__ void __launch_bounds__(kBlasThreads) site_batch_kernel(Op op, int vh, int lognp, double *partials,
                                                                  unsigned int *counter, Gate gate)
{
    static_assert(Op::NRED <= kBatchMaxRed, "partials hold kBatchMaxRed sums per (block, RHS)");
    if (gate.closed()) return;
    constexpr int NR = Op::NRED > 0 ? Op::NRED : 1;
    const int np = 1 << lognp, nb = 2 * np;
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    const int q = tid & (np - 1);
    double acc[2 * NR];
#pragma unroll
    for (int k = 0; k < 2 * NR; ++k) acc[k] = 0.0;
    const long total = (long)vh << lognp;
    for (long i = tid; i < total; i += (long)gridDim.x * blockDim.x) op.site((int)(i >> lognp), q, acc);
    if constexpr (Op::NRED > 0) {
        __shared__ double smem[kBlasThreads / 32][kMaxBatch][NR];
        __shared__ bool last;
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
        for (int k = 0; k < 2 * NR; ++k) {
            double x = acc[k];
            for (int o = 16; o >= np; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
            acc[k] = x;
        }
        if (lane < np)
#pragma unroll
            for (int k = 0; k < NR; ++k) {
                smem[warp][2 * lane][k] = acc[k];
                smem[warp][2 * lane + 1][k] = acc[NR + k];
            }
        __syncthreads();
        if (threadIdx.x < nb) {
            for (int k = 0; k < NR; ++k) {
                double s = 0.0;
                for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += smem[w][threadIdx.x][k];
                partials[((size_t)blockIdx.x * kMaxBatch + threadIdx.x) * NR + k] = s;
            }
            __threadfence();  // every writer makes its partial sums visible device-wide
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            const unsigned int ticket = atomicAdd(counter, 1u);
            last = (ticket == gridDim.x - 1);
        }
        __syncthreads();
        if (last) {
            __threadfence();
            // every thread sums a fixed chunk of the blocks for one RHS (thread = chunk * nb + r),
            // then thread r adds the chunks in order: deterministic, and the block partials are
            // read by all threads instead of nb
            const int nchunk = blockDim.x / nb, G = gridDim.x;
            double(*red)[NR] = &smem[0][0];  // [nchunk * nb][NR], the same storage
            if ((int)threadIdx.x < nchunk * nb) {
                const int r = threadIdx.x % nb, ch = threadIdx.x / nb;
                const int b0 = (int)((long)ch * G / nchunk), b1 = (int)((long)(ch + 1) * G / nchunk);
                double part[NR];
#pragma unroll
                for (int k = 0; k < NR; ++k) part[k] = 0.0;
                for (int b = b0; b < b1; ++b) {
                    const double *src = partials + ((size_t)b * kMaxBatch + r) * NR;
#pragma unroll
                    for (int k = 0; k < NR; ++k) part[k] += __ldcg(src + k);
                }
#pragma unroll
                for (int k = 0; k < NR; ++k) red[threadIdx.x][k] = part[k];
            }
            __syncthreads();
            if (threadIdx.x < nb) {
                double tot[NR];
#pragma unroll
                for (int k = 0; k < NR; ++k) {
                    double s = 0.0;
                    for (int ch = 0; ch < nchunk; ++ch) s += red[ch * nb + threadIdx.x][k];
                    tot[k] = s;
                }
                op.finalize(threadIdx.x, tot);
            }
            __syncthreads();
            if (threadIdx.x == 0) {
                op.finalize_all();
                *counter = 0u;
            }
        }
    }
}

// ------------------------------------------------------ batched CG state ---
// A slot whose recursive residual fell by delta2 (or reached eps) parks: it leaves the
// iteration (active = 0, need_update = 1) while the others go on, and the captured
// loop pauses for the host's FP64 reliable updates once park_limit slots are parked or
// none is left running.
struct BatchCGState {
    int pause;                 // gates every captured kernel
    int iter, max_iter, nb;
    int park_limit;
    double delta2;
    double rr[kMaxBatch], rr_prev[kMaxBatch], rr_max[kMaxBatch], eps[kMaxBatch], beta[kMaxBatch];
    double2 alpha[kMaxBatch];
    int active[kMaxBatch];     // 0: converged and frozen
    int converged[kMaxBatch];  // the recursion's residual reached eps
    int need_update[kMaxBatch];
    int its[kMaxBatch];        // iterations each slot took part in
    int failed;
    double2 rho[kMaxBatch], omega[kMaxBatch], bbeta[kMaxBatch];  // BiCGStab only
    int restart[kMaxBatch];                    // broke down: restart at the update
                                               // (2: non-finite, drop the FP32 accumulator)
    int last_update_its[kMaxBatch];            // its at the last reliable update
    // the slot's FP32 solution accumulator counts as zero in the next update pass (it was
    // folded into the FP64 solution or dropped, or the slot took a new source), which
    // spares a pass that would clear one lane of the pair layout
    int x_reset[kMaxBatch];
};

LYM_D cx<double> as_cx2(double2 z) { return cx<double>{z.x, z.y}; }

// a slot gets a reliable update at least every kForcedUpdateIts of its iterations, so a
// stagnating recursion still reaches the host's progress check
constexpr int kForcedUpdateIts = 200;

// finalize_all of the step that closes an iteration: counts it and pauses the captured
// loop at the iteration limit, when no slot is left running, or when park_limit slots
// wait for their reliable update
LYM_D void batch_iteration_done(BatchCGState *s)
{
    s->iter += 1;
    int parked = 0, running = 0;
    for (int r = 0; r < s->nb; ++r) {
        parked += s->need_update[r];
        running += s->active[r];
    }
    if (s->iter >= s->max_iter || running == 0 || parked >= s->park_limit) s->pause = 1;
}

// Output of one pair, written one component at a time: FP32 words go out at once, FP16
// words wait for the whole site (the per-site norm needs every component).
template <class B> struct PairOut;
template <> struct PairOut<BatchF> {
    BatchF b;
    int h, q;
    LYM_D void put(int c, cx<double> x, cx<double> y) { b.put(h, q, c, x, y); }
    LYM_D void finish() {}
};
template <> struct PairOut<BatchH> {
    BatchH b;
    int h, q;
    c2 buf[12];
    LYM_D void put(int c, cx<double> x, cx<double> y)
    {
        buf[c] = c2{make_float2((float)x.re, (float)y.re), make_float2((float)x.im, (float)y.im)};
    }
    LYM_D void finish() { b.store(h, q, buf); }
};
template <class B> LYM_D PairOut<B> pair_out(const B &b, int h, int q) { return PairOut<B>{b, h, q}; }

// acc += conj(a) b (re, im) and |a|^2 helpers for single components
LYM_D void dot1(cx<double> a, cx<double> b, double &re, double &im)
{
    re += a.re * b.re + a.im * b.im;
    im += a.re * b.im - a.im * b.re;
}
LYM_D double nrm1(cx<double> a) { return a.re * a.re + a.im * a.im; }

// alpha_r = rr_r / <p_r, A p_r>
template <class SP, class SAp> struct OpBAlpha {
    static constexpr int NRED = 2;
    SP p;
    SAp ap;
    BatchCGState *s;
    LYM_D void site(int h, int q, double *acc) const
    {
        const bool a0 = s->active[2 * q] != 0, a1 = s->active[2 * q + 1] != 0;
        if (!a0 && !a1) return;
#pragma unroll 2
        for (int c = 0; c < 12; ++c) {
            cx<double> x0, x1, y0, y1;
            p.get(h, q, c, x0, x1);
            ap.get(h, q, c, y0, y1);
            if (a0) dot1(x0, y0, acc[0], acc[1]);
            if (a1) dot1(x1, y1, acc[2], acc[3]);
        }
    }
    LYM_D void finalize(int r, const double *t) const
    {
        if (s->active[r]) s->alpha[r] = cdiv(make_double2(s->rr[r], 0.0), make_double2(t[0], t[1]));
    }
    LYM_D void finalize_all() const {}
};

// x_r += alpha_r p_r, res_r -= alpha_r A p_r, rr_r = |res_r|^2 and the convergence /
// reliable-update decisions
template <class SX, class SP, class SR, class SAp> struct OpBUpdate {
    static constexpr int NRED = 1;
    SX x;
    SP p;
    SR rv;
    SAp ap;
    BatchCGState *s;
    LYM_D void site(int h, int q, double *acc) const
    {
        const bool act[2] = {s->active[2 * q] != 0, s->active[2 * q + 1] != 0};
        if (!act[0] && !act[1]) return;
        const cx<double> al[2] = {as_cx2(s->alpha[2 * q]), as_cx2(s->alpha[2 * q + 1])};
        const bool xr[2] = {s->x_reset[2 * q] != 0, s->x_reset[2 * q + 1] != 0};
        auto xo = pair_out(x, h, q);
        auto ro = pair_out(rv, h, q);
#pragma unroll 2
        for (int c = 0; c < 12; ++c) {
            cx<double> xv[2], pv[2], res[2], av[2];
            x.get(h, q, c, xv[0], xv[1]);
            p.get(h, q, c, pv[0], pv[1]);
            rv.get(h, q, c, res[0], res[1]);
            ap.get(h, q, c, av[0], av[1]);
#pragma unroll
            for (int l = 0; l < 2; ++l) {
                if (!act[l]) continue;
                if (xr[l]) xv[l] = cx<double>{0.0, 0.0};
                fma_c(xv[l], al[l], pv[l]);
                res[l] = res[l] - al[l] * av[l];
                acc[l] += nrm1(res[l]);
            }
            xo.put(c, xv[0], xv[1]);
            ro.put(c, res[0], res[1]);
        }
        xo.finish();
        ro.finish();
    }
    LYM_D void finalize(int r, const double *t) const
    {
        if (!s->active[r]) return;
        s->x_reset[r] = 0;
        s->its[r] += 1;
        const double rr_new = t[0];
        s->rr_prev[r] = s->rr[r];
        s->beta[r] = rr_new / s->rr[r];
        s->rr[r] = rr_new;
        if (rr_new > s->rr_max[r]) s->rr_max[r] = rr_new;
        if (!(rr_new <= 1e300)) {  // non-finite: this RHS leaves the iteration; the host restarts
            s->restart[r] = 2;     // it from its FP64 solution or stops it (the others go on)
            s->need_update[r] = 1;
            s->active[r] = 0;
        } else if (rr_new < s->eps[r]) {
            s->converged[r] = 1;
            s->need_update[r] = 1;
            s->active[r] = 0;
        } else if (rr_new < s->delta2 * s->rr_max[r]) {
            s->need_update[r] = 1;
            s->active[r] = 0;
        }
    }
    LYM_D void finalize_all() const { batch_iteration_done(s); }
};

// p_r = res_r + beta_r p_r for the active RHS that need no reliable update
template <class SP, class SR> struct OpBDirection {
    static constexpr int NRED = 0;
    SP p;
    SR rv;
    BatchCGState *s;
    LYM_D void site(int h, int q, double *) const
    {
        bool go[2];
#pragma unroll
        for (int l = 0; l < 2; ++l) go[l] = s->active[2 * q + l] && !s->need_update[2 * q + l];
        if (!go[0] && !go[1]) return;
        const double b[2] = {s->beta[2 * q], s->beta[2 * q + 1]};
        auto po = pair_out(p, h, q);
#pragma unroll 2
        for (int c = 0; c < 12; ++c) {
            cx<double> pv[2], res[2];
            p.get(h, q, c, pv[0], pv[1]);
            rv.get(h, q, c, res[0], res[1]);
#pragma unroll
            for (int l = 0; l < 2; ++l)
                if (go[l]) pv[l] = res[l] + b[l] * pv[l];
            po.put(c, pv[0], pv[1]);
        }
        po.finish();
    }
    LYM_D void finalize(int, const double *) const {}
    LYM_D void finalize_all() const {}
};

// -------------------------------------------------- batched BiCGStab ops ---
// One iteration of BiCGStab on the Schur operator S (no gamma5), per RHS r:
//   v = S p;  alpha = rho / <rhat, v>;  s = r - alpha v;  t = S s;
//   omega = <t, s> / |t|^2;  x += alpha p + omega s;  r = s - omega t;
//   rho' = <rhat, r>;  beta = (rho' / rho) (alpha / omega);  p = r + beta (p - omega v)
// (BiConjugateGradient::solve, inverters/BiConjugateGradient.cpp:321-507, with the
// scalars kept per RHS in FP64 and the vectors in the batch precisions).

LYM_D double2 as_d2(cx<double> z) { return make_double2(z.re, z.im); }
LYM_D cx<double> as_cx(double2 z) { return cx<double>{z.x, z.y}; }

// omega_r = <t_r, s_r> / |t_r|^2;  rho'_r = <rhat_r, r'_r> = <rhat_r, s_r> - omega_r <rhat_r, t_r>;
// beta_r = (rho'_r / rho_r) (alpha_r / omega_r).  A zero |t|^2 or rho' marks the slot for a
// restart (the update parks it).
// omega, rho' and beta of RHS r from t[7] = <t,s>, |t|^2, <rhat,s>, <rhat,t>
LYM_D void omega_finalize(BatchCGState *s, int r, const double *t)
{
    if (!s->active[r]) return;
    const double2 om = t[2] > 0.0 ? make_double2(t[0] / t[2], t[1] / t[2]) : make_double2(0.0, 0.0);
    const double2 rho_new = csub(make_double2(t[3], t[4]), cmul(om, make_double2(t[5], t[6])));
    const bool stalled = (om.x == 0.0 && om.y == 0.0) || (rho_new.x == 0.0 && rho_new.y == 0.0);
    s->omega[r] = om;
    s->bbeta[r] = stalled ? make_double2(0.0, 0.0) : cmul(cdiv(rho_new, s->rho[r]), cdiv(s->alpha[r], om));
    s->rho[r] = rho_new;
    if (stalled) s->restart[r] = 1;
}

template <class ST, class SS, class SRh> struct OpBBOmega {
    static constexpr int NRED = 7;
    ST tv;
    SS sv;
    SRh rh;
    BatchCGState *s;
    LYM_D void site(int h, int q, double *acc) const
    {
        const bool act[2] = {s->active[2 * q] != 0, s->active[2 * q + 1] != 0};
        if (!act[0] && !act[1]) return;
#pragma unroll 2
        for (int c = 0; c < 12; ++c) {
            cx<double> t[2], sw[2], hv[2];
            tv.get(h, q, c, t[0], t[1]);
            sv.get(h, q, c, sw[0], sw[1]);
            rh.get(h, q, c, hv[0], hv[1]);
#pragma unroll
            for (int l = 0; l < 2; ++l) {
                if (!act[l]) continue;
                double *a = acc + 7 * l;
                dot1(t[l], sw[l], a[0], a[1]);
                a[2] += nrm1(t[l]);
                dot1(hv[l], sw[l], a[3], a[4]);
                dot1(hv[l], t[l], a[5], a[6]);
            }
        }
    }
    LYM_D void finalize(int r, const double *t) const { omega_finalize(s, r, t); }
    LYM_D void finalize_all() const {}
};

// x_r += alpha_r p_r + omega_r s_r;  r_r = s_r - omega_r t_r;  p_r = r_r + beta_r (p_r - omega_r v_r);
// |r_r|^2 and <what_r, p_r> (what = S^+ rhat, so that <rhat, S p> of the next iteration is
// known now: alpha_r = rho_r / <what_r, p_r>), and the convergence / reliable-update decisions
template <class SX, class SP, class SS, class ST, class SV, class SR, class SW> struct OpBBUpdate {
    static constexpr int NRED = 3;
    SX x;
    SP p;
    SS sv;
    ST tv;
    SV v;
    SR rv;
    SW wh;
    BatchCGState *s;
    LYM_D void site(int h, int q, double *acc) const
    {
        const bool act[2] = {s->active[2 * q] != 0, s->active[2 * q + 1] != 0};
        if (!act[0] && !act[1]) return;
        const bool idle = !act[0] || !act[1];
        cx<double> al[2], om[2], be[2];
#pragma unroll
        for (int l = 0; l < 2; ++l) {
            al[l] = as_cx(s->alpha[2 * q + l]);
            om[l] = as_cx(s->omega[2 * q + l]);
            be[l] = as_cx(s->bbeta[2 * q + l]);
        }
        const bool xr[2] = {s->x_reset[2 * q] != 0, s->x_reset[2 * q + 1] != 0};
        auto xo = pair_out(x, h, q);
        auto ro = pair_out(rv, h, q);
        auto po = pair_out(p, h, q);
#pragma unroll 2
        for (int c = 0; c < 12; ++c) {
            cx<double> xv[2], pv[2], sw[2], tw[2], vv[2], rr[2], ww[2];
            x.get(h, q, c, xv[0], xv[1]);
            p.get(h, q, c, pv[0], pv[1]);
            sv.get(h, q, c, sw[0], sw[1]);
            tv.get(h, q, c, tw[0], tw[1]);
            v.get(h, q, c, vv[0], vv[1]);
            wh.get(h, q, c, ww[0], ww[1]);
            if (idle) rv.get(h, q, c, rr[0], rr[1]);  // an idle lane keeps its residual
#pragma unroll
            for (int l = 0; l < 2; ++l) {
                if (!act[l]) continue;
                if (xr[l]) xv[l] = cx<double>{0.0, 0.0};
                fma_c(xv[l], al[l], pv[l]);
                fma_c(xv[l], om[l], sw[l]);
                rr[l] = sw[l] - om[l] * tw[l];
                pv[l] = rr[l] + be[l] * (pv[l] - om[l] * vv[l]);
                acc[3 * l] += nrm1(rr[l]);
                dot1(ww[l], pv[l], acc[3 * l + 1], acc[3 * l + 2]);
            }
            xo.put(c, xv[0], xv[1]);
            ro.put(c, rr[0], rr[1]);
            po.put(c, pv[0], pv[1]);
        }
        xo.finish();
        ro.finish();
        po.finish();
    }
    LYM_D void finalize(int r, const double *t) const
    {
        if (!s->active[r]) return;
        s->x_reset[r] = 0;
        s->its[r] += 1;
        const double rr_new = t[0];
        s->rr_prev[r] = s->rr[r];
        s->rr[r] = rr_new;
        if (rr_new > s->rr_max[r]) s->rr_max[r] = rr_new;
        const bool breakdown = t[1] == 0.0 && t[2] == 0.0;
        if (!(rr_new <= 1e300)) {  // non-finite: the recursion broke down on this RHS; its FP32
            s->restart[r] = 2;     // accumulator is discarded and it restarts from its FP64 x
            s->need_update[r] = 1;
            s->active[r] = 0;
        } else if (rr_new < s->eps[r]) {
            s->converged[r] = 1;
            s->need_update[r] = 1;
            s->active[r] = 0;
        } else if (s->restart[r] || breakdown || rr_new < s->delta2 * s->rr_max[r] ||
                   s->its[r] - s->last_update_its[r] >= kForcedUpdateIts) {
            if (breakdown) s->restart[r] = 1;
            s->need_update[r] = 1;
            s->active[r] = 0;
        } else {
            s->alpha[r] = cdiv(s->rho[r], make_double2(t[1], t[2]));
        }
    }
    LYM_D void finalize_all() const { batch_iteration_done(s); }
};

}  // namespace lym
