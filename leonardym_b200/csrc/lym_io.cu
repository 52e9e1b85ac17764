// Gauge-configuration files as LeonardYM writes and reads them (io/OutputSweep.cpp:32-440,
// starters/ReadStartGaugeConfiguration.cpp:36-480), host code only.  Values are XDR
// (RFC 4506): 32-bit big-endian integers and IEEE-754 floats, 64-bit big-endian doubles;
// the encoding is written out here because the image has no XDR library.
//
// Links are fundamental gauge links in the reference's raw layout, double[V][4][N][N][2]
// with [site][mu][j][i] = U_mu(site)(i, j) (an Eigen column-major matrix per link) and site
// t + Lt (z + Lz (y + Ly x)).
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/lym_b200.h"

namespace {

using cplx = std::complex<double>;

struct XdrIn {
    std::vector<unsigned char> buf;
    size_t pos = 0;
    bool ok = true;
    bool load(const std::string &path)
    {
        FILE *f = fopen(path.c_str(), "rb");
        if (!f) return false;
        fseek(f, 0, SEEK_END);
        const long n = ftell(f);
        fseek(f, 0, SEEK_SET);
        buf.resize(n > 0 ? (size_t)n : 0);
        const size_t got = n > 0 ? fread(buf.data(), 1, buf.size(), f) : 0;
        fclose(f);
        return got == buf.size();
    }
    uint32_t u32()
    {
        if (pos + 4 > buf.size()) {
            ok = false;
            return 0;
        }
        const uint32_t v = (uint32_t)buf[pos] << 24 | (uint32_t)buf[pos + 1] << 16 | (uint32_t)buf[pos + 2] << 8 |
                           (uint32_t)buf[pos + 3];
        pos += 4;
        return v;
    }
    int i32() { return (int)u32(); }
    float f32()
    {
        const uint32_t v = u32();
        float f;
        std::memcpy(&f, &v, 4);
        return f;
    }
    double f64()
    {
        const uint64_t hi = u32(), lo = u32();
        const uint64_t v = hi << 32 | lo;
        double d;
        std::memcpy(&d, &v, 8);
        return d;
    }
};

struct XdrOut {
    std::vector<unsigned char> buf;
    void u32(uint32_t v)
    {
        buf.push_back((unsigned char)(v >> 24));
        buf.push_back((unsigned char)(v >> 16));
        buf.push_back((unsigned char)(v >> 8));
        buf.push_back((unsigned char)v);
    }
    void i32(int v) { u32((uint32_t)v); }
    void f32(float f)
    {
        uint32_t v;
        std::memcpy(&v, &f, 4);
        u32(v);
    }
    void f64(double d)
    {
        uint64_t v;
        std::memcpy(&v, &d, 8);
        u32((uint32_t)(v >> 32));
        u32((uint32_t)v);
    }
    bool save(const std::string &path) const
    {
        FILE *f = fopen(path.c_str(), "wb");
        if (!f) return false;
        const bool ok = fwrite(buf.data(), 1, buf.size(), f) == buf.size();
        return fclose(f) == 0 && ok;
    }
};

struct Links {
    double *p;
    int n;
    cplx get(long site, int mu, int i, int j) const
    {
        const double *e = p + ((((size_t)site * 4 + mu) * n + j) * n + i) * 2;
        return cplx(e[0], e[1]);
    }
    void set(long site, int mu, int i, int j, cplx v) const
    {
        double *e = p + ((((size_t)site * 4 + mu) * n + j) * n + i) * 2;
        e[0] = v.real();
        e[1] = v.imag();
    }
};

long lex(const int d[4], int x, int y, int z, int t) { return t + (long)d[3] * (z + (long)d[2] * (y + (long)d[1] * x)); }
long volume(const int d[4]) { return (long)d[0] * d[1] * d[2] * d[3]; }
double absq(cplx z) { return z.real() * z.real() + z.imag() * z.imag(); }

std::string leonard_base(const char *dir, const char *name, int number)
{
    return std::string(dir) + name + "_" + std::to_string(number);
}
std::string muenster_su2_path(const char *dir, const char *name, int number)
{
    return std::string(dir) + "0:" + std::to_string(number) + ":" + name;
}
std::string muenster_su3_path(const char *dir, const char *name, int number)
{
    return std::string(dir) + name + ".config-" + std::to_string(number);
}

// ReadStartGaugeConfiguration.cpp:51-130 (leonard_format): descriptor, then per processor
// file: per site x, y, z, t and U(i, j) row by row as XDR double pairs
int read_leonard(const int d[4], int nc, const char *dir, const char *name, int number, Links U, double *plaq)
{
    std::ifstream desc(leonard_base(dir, name, number) + ".descriptor.txt");
    if (!desc) return LYM_ERR_NOT_FOUND;
    int g[4], pg[4], nproc = 0;
    long localsize = 0;
    double p = 0.0;
    desc >> g[0] >> g[1] >> g[2] >> g[3] >> pg[0] >> pg[1] >> pg[2] >> pg[3] >> nproc >> localsize >> p;
    if (!desc) return LYM_ERR_ARGUMENT;
    for (int k = 0; k < 4; ++k)
        if (g[k] != d[k]) return LYM_ERR_ARGUMENT;  // "Different lattice size in reading configuration!"
    if (nproc < 1 || localsize < 1) return LYM_ERR_ARGUMENT;
    std::vector<char> seen(volume(d), 0);
    for (int proc = 0; proc < nproc; ++proc) {
        XdrIn in;
        if (!in.load(leonard_base(dir, name, number) + "_" + std::to_string(proc) + ".txt")) return LYM_ERR_NOT_FOUND;
        for (long k = 0; k < localsize; ++k) {
            const int x = in.i32(), y = in.i32(), z = in.i32(), t = in.i32();
            const bool inside = x >= 0 && x < d[0] && y >= 0 && y < d[1] && z >= 0 && z < d[2] && t >= 0 && t < d[3];
            const long site = inside ? lex(d, x, y, z, t) : -1;
            for (int mu = 0; mu < 4; ++mu)
                for (int i = 0; i < nc; ++i)
                    for (int j = 0; j < nc; ++j) {
                        const double re = in.f64(), im = in.f64();
                        if (site >= 0) U.set(site, mu, i, j, cplx(re, im));
                    }
            if (site >= 0) seen[site] = 1;
            if (!in.ok) return LYM_ERR_ARGUMENT;
        }
    }
    for (char s : seen)
        if (!s) return LYM_ERR_ARGUMENT;  // a site no processor file held
    if (plaq) *plaq = p;
    return LYM_OK;
}

// OutputSweep.cpp:32-85 for one process (pgrid 1 1 1 1)
int write_leonard(const int d[4], int nc, const char *dir, const char *name, int number, Links U, double plaq)
{
    XdrOut out;
    for (int x = 0; x < d[0]; ++x)
        for (int y = 0; y < d[1]; ++y)
            for (int z = 0; z < d[2]; ++z)
                for (int t = 0; t < d[3]; ++t) {
                    const long site = lex(d, x, y, z, t);
                    out.i32(x);
                    out.i32(y);
                    out.i32(z);
                    out.i32(t);
                    for (int mu = 0; mu < 4; ++mu)
                        for (int i = 0; i < nc; ++i)
                            for (int j = 0; j < nc; ++j) {
                                const cplx v = U.get(site, mu, i, j);
                                out.f64(v.real());
                                out.f64(v.imag());
                            }
                }
    if (!out.save(leonard_base(dir, name, number) + "_0.txt")) return LYM_ERR_NOT_FOUND;
    std::ofstream desc(leonard_base(dir, name, number) + ".descriptor.txt");
    if (!desc) return LYM_ERR_NOT_FOUND;
    desc << d[0] << " " << d[1] << " " << d[2] << " " << d[3] << std::endl;
    desc << 1 << " " << 1 << " " << 1 << " " << 1 << std::endl;
    desc << 1 << std::endl;
    desc << volume(d) << std::endl;
    desc << std::setprecision(13) << plaq << std::endl;
    return desc ? LYM_OK : LYM_ERR_NOT_FOUND;
}

// SU(2) muenster_format (ReadStartGaugeConfiguration.cpp:131-300): sites with x fastest, per
// link U^+(0,0), U^+(0,1) as XDR floats, then the trailer (plaquette, correction factor,
// smallest eigenvalue, beta, kappas (all but the last negative), alphas, epsilon / lambda
// pairs, sweep, 5 polynomial orders per kappa, the extents, lvrc)
int read_muenster_su2(const int d[4], const char *dir, const char *name, int number, Links U, double *plaq)
{
    XdrIn in;
    if (!in.load(muenster_su2_path(dir, name, number))) return LYM_ERR_NOT_FOUND;
    for (int t = 0; t < d[3]; ++t)
        for (int z = 0; z < d[2]; ++z)
            for (int y = 0; y < d[1]; ++y)
                for (int x = 0; x < d[0]; ++x) {
                    const long site = lex(d, x, y, z, t);
                    for (int mu = 0; mu < 4; ++mu)
                        for (int ii = 0; ii < 2; ++ii) {
                            const float a = in.f32(), b = in.f32();
                            const cplx c(a, b);
                            U.set(site, mu, 0, ii, ii == 0 ? std::conj(c) : -c);
                            U.set(site, mu, 1, ii == 0 ? 1 : 0, ii == 0 ? c : std::conj(c));
                        }
                }
    if (!in.ok) return LYM_ERR_ARGUMENT;  // "read error for gauge fields"
    const float p = in.f32();
    in.f32();
    in.f32();
    in.f32();  // beta
    int nferm = 0;
    for (float kappa = -1.0f; kappa < 0.0f && in.ok;) {
        kappa = in.f32();
        ++nferm;
    }
    for (int k = 0; k < nferm; ++k) in.f32();
    for (int k = 0; k < nferm; ++k) in.f32(), in.f32();
    in.i32();  // sweep
    for (int k = 0; k < 5 * nferm; ++k) in.i32();
    int lat[4];
    for (int k = 0; k < 4; ++k) lat[k] = in.i32();
    in.i32();
    if (!in.ok) return LYM_ERR_ARGUMENT;
    for (int k = 0; k < 4; ++k)
        if (lat[k] != d[k]) return LYM_ERR_ARGUMENT;  // "Lattice size is different"
    if (plaq) *plaq = p;
    return LYM_OK;
}

// OutputSweep.cpp:87-285 for one process: one kappa, zero alphas / epsilons / lambdas /
// polynomial orders, lvrc 0
int write_muenster_su2(const int d[4], const char *dir, const char *name, int number, Links U, double plaq, double beta,
                       double kappa)
{
    XdrOut out;
    for (int t = 0; t < d[3]; ++t)
        for (int z = 0; z < d[2]; ++z)
            for (int y = 0; y < d[1]; ++y)
                for (int x = 0; x < d[0]; ++x) {
                    const long site = lex(d, x, y, z, t);
                    for (int mu = 0; mu < 4; ++mu) {
                        // U^+(0,0) = conj U(0,0), U^+(0,1) = conj U(1,0)
                        const cplx a = std::conj(U.get(site, mu, 0, 0)), b = std::conj(U.get(site, mu, 1, 0));
                        out.f32((float)a.real());
                        out.f32((float)a.imag());
                        out.f32((float)b.real());
                        out.f32((float)b.imag());
                    }
                }
    out.f32((float)plaq);
    out.f32(0.0f);
    out.f32(0.0f);
    out.f32((float)beta);
    out.f32((float)kappa);
    out.f32(0.0f);  // alpha
    out.f32(0.0f);  // epsilon
    out.f32(0.0f);  // lambda
    out.i32(number);
    for (int k = 0; k < 5; ++k) out.i32(0);
    for (int k = 0; k < 4; ++k) out.i32(d[k]);
    out.i32(0);
    return out.save(muenster_su2_path(dir, name, number)) ? LYM_OK : LYM_ERR_NOT_FOUND;
}

// SU(3) muenster_format (ReadStartGaugeConfiguration.cpp:300-480): per link the first two
// columns of U^* as XDR float pairs (row by row), the columns re-orthonormalised and the
// third column their conjugated cross product; trailer: extents, beta, c1, plaquette (doubles)
int read_muenster_su3(const int d[4], const char *dir, const char *name, int number, Links U, double *plaq)
{
    XdrIn in;
    if (!in.load(muenster_su3_path(dir, name, number))) return LYM_ERR_NOT_FOUND;
    for (int t = 0; t < d[3]; ++t)
        for (int z = 0; z < d[2]; ++z)
            for (int y = 0; y < d[1]; ++y)
                for (int x = 0; x < d[0]; ++x) {
                    const long site = lex(d, x, y, z, t);
                    for (int mu = 0; mu < 4; ++mu) {
                        cplx m[3][3];
                        for (int ii = 0; ii < 3; ++ii)
                            for (int jj = 0; jj < 2; ++jj) {
                                const float a = in.f32(), b = in.f32();
                                m[ii][jj] = cplx(a, -b);
                            }
                        {
                            const cplx s = 1.0 / std::sqrt(absq(m[0][0]) + absq(m[1][0]) + absq(m[2][0]));
                            for (int ii = 0; ii < 3; ++ii) m[ii][0] *= s;
                        }
                        {
                            const cplx s = m[0][1] * std::conj(m[0][0]) + m[1][1] * std::conj(m[1][0]) +
                                           m[2][1] * std::conj(m[2][0]);
                            for (int ii = 0; ii < 3; ++ii) m[ii][1] -= s * m[ii][0];
                        }
                        {
                            const cplx s = 1.0 / std::sqrt(absq(m[0][1]) + absq(m[1][1]) + absq(m[2][1]));
                            for (int ii = 0; ii < 3; ++ii) m[ii][1] *= s;
                        }
                        m[0][2] = std::conj(m[1][0]) * std::conj(m[2][1]) - std::conj(m[2][0]) * std::conj(m[1][1]);
                        m[1][2] = std::conj(m[2][0]) * std::conj(m[0][1]) - std::conj(m[0][0]) * std::conj(m[2][1]);
                        m[2][2] = std::conj(m[0][0]) * std::conj(m[1][1]) - std::conj(m[1][0]) * std::conj(m[0][1]);
                        for (int ii = 0; ii < 3; ++ii)
                            for (int jj = 0; jj < 3; ++jj) U.set(site, mu, ii, jj, m[ii][jj]);
                    }
                }
    if (!in.ok) return LYM_ERR_ARGUMENT;
    int lat[4];
    for (int k = 0; k < 4; ++k) lat[k] = in.i32();
    in.f64();  // beta
    in.f64();  // c1
    if (!in.ok) return LYM_ERR_ARGUMENT;
    for (int k = 0; k < 4; ++k)
        if (lat[k] != d[k]) return LYM_ERR_ARGUMENT;
    const double p = in.f64();
    if (plaq) *plaq = in.ok ? p : NAN;  // "no temporal plaquette value found"
    return LYM_OK;
}

// OutputSweep.cpp:286-440 for one process
int write_muenster_su3(const int d[4], const char *dir, const char *name, int number, Links U, double plaq, double beta)
{
    XdrOut out;
    for (int t = 0; t < d[3]; ++t)
        for (int z = 0; z < d[2]; ++z)
            for (int y = 0; y < d[1]; ++y)
                for (int x = 0; x < d[0]; ++x) {
                    const long site = lex(d, x, y, z, t);
                    for (int mu = 0; mu < 4; ++mu)
                        for (int ii = 0; ii < 3; ++ii)
                            for (int jj = 0; jj < 2; ++jj) {
                                const cplx v = U.get(site, mu, ii, jj);
                                out.f32((float)v.real());
                                out.f32((float)-v.imag());
                            }
                }
    for (int k = 0; k < 4; ++k) out.i32(d[k]);
    out.f64((double)(float)beta);
    out.f64(-1.0 / 12.0);
    out.f64(plaq);
    return out.save(muenster_su3_path(dir, name, number)) ? LYM_OK : LYM_ERR_NOT_FOUND;
}

bool valid(const int d[4], int nc, const char *dir, const char *name, const void *links)
{
    if (!d || !dir || !name || !links || (nc != 2 && nc != 3)) return false;
    for (int k = 0; k < 4; ++k)
        if (d[k] < 1) return false;
    return true;
}

}  // namespace

extern "C" {

int lym_gauge_file_read(int format, const int dims[4], int nc, const char *directory, const char *name, int number,
                        double *links, double *plaquette)
{
    if (!valid(dims, nc, directory, name, links)) return LYM_ERR_ARGUMENT;
    const Links U{links, nc};
    try {
        if (format == LYM_GAUGE_LEONARD) return read_leonard(dims, nc, directory, name, number, U, plaquette);
        if (format == LYM_GAUGE_MUENSTER)
            return nc == 2 ? read_muenster_su2(dims, directory, name, number, U, plaquette)
                           : read_muenster_su3(dims, directory, name, number, U, plaquette);
    } catch (const std::bad_alloc &) {
        return LYM_ERR_MEMORY;
    }
    return LYM_ERR_ARGUMENT;
}

int lym_gauge_file_write(int format, const int dims[4], int nc, const double *links, const char *directory,
                         const char *name, int number, double plaquette, double beta, double kappa)
{
    if (!valid(dims, nc, directory, name, links)) return LYM_ERR_ARGUMENT;
    const Links U{const_cast<double *>(links), nc};
    try {
        if (format == LYM_GAUGE_LEONARD) return write_leonard(dims, nc, directory, name, number, U, plaquette);
        if (format == LYM_GAUGE_MUENSTER)
            return nc == 2 ? write_muenster_su2(dims, directory, name, number, U, plaquette, beta, kappa)
                           : write_muenster_su3(dims, directory, name, number, U, plaquette, beta);
    } catch (const std::bad_alloc &) {
        return LYM_ERR_MEMORY;
    }
    return LYM_ERR_ARGUMENT;
}

}  // extern "C"
