/*
 * formats.cpp -- mesh / Jacobian stream-binary I/O, validation and the
 * seeded structured-mesh generator (host C++, no device code).
 *
 * Layouts (little-endian, no Fortran record markers, access='stream'):
 *   mesh      int32 [nvar nelem nintface eftot nline nlineelem]
 *             epoint[nelem+1] ef[eftot] fc[2*nintface] linesize[nline]
 *             linepoint[nline+1] lines[nlineelem] lineface[nlineelem]
 *             (src/F90/read_mesh_data.F90:28-35, data/ex05/line.input.data)
 *             all indices 1-based on disk, shifted to 0-based on load
 *             (src/F90/read_mesh_data.F90:41-64).
 *   jacobian  int32 [nvar nelem nintface], then FP64 jacD[nvar^2*nelem]
 *             jacO1[nvar^2*nintface] jacO2[..] rhs[nvar*nelem] U0[..],
 *             starting at byte 12 (src/F90/read_jacobian_data.F90:26-31).
 */
#include "tbs_internal.hxx"

#include <cstdio>
#include <cstring>
#include <string>
#include <vector>
#include <sys/stat.h>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace tbs {

static thread_local std::string g_thread_error;

void set_thread_error(const std::string &msg) { g_thread_error = msg; }
const char *thread_error() { return g_thread_error.c_str(); }

static int fail(int code, const std::string &msg) {
    set_thread_error(msg);
    return code;
}

static long long file_size(const char *path) {
    struct stat st;
    if (stat(path, &st) != 0) return -1;
    return (long long)st.st_size;
}

long long mesh_file_bytes(const int hdr[6]) {
    const long long nelem = hdr[1], nint = hdr[2], eftot = hdr[3];
    const long long nline = hdr[4], nle = hdr[5];
    return 4LL * (6 + (nelem + 1) + eftot + 2 * nint + nline + (nline + 1) + 2 * nle);
}

long long jacobian_file_bytes(const int hdr[3]) {
    const long long nv = hdr[0], nelem = hdr[1], nint = hdr[2];
    return 12LL + 8LL * (nv * nv * nelem + 2 * nv * nv * nint + 2 * nv * nelem);
}

/* fread of n items that reports short reads (the reference ignores the
 * fread result, src/Mesh.cxx:24 / src/Jacobian.cxx:22). */
template <typename T>
static bool read_n(FILE *fp, T *dst, size_t n) {
    const size_t chunk = size_t(1) << 24;
    size_t done = 0;
    while (done < n) {
        size_t want = (n - done < chunk) ? n - done : chunk;
        size_t got = fread(dst + done, sizeof(T), want, fp);
        if (got != want) return false;
        done += got;
    }
    return true;
}

template <typename T>
static bool write_n(FILE *fp, const T *src, size_t n) {
    const size_t chunk = size_t(1) << 24;
    size_t done = 0;
    while (done < n) {
        size_t want = (n - done < chunk) ? n - done : chunk;
        if (fwrite(src + done, sizeof(T), want, fp) != want) return false;
        done += want;
    }
    return true;
}

static bool header_sane(const int hdr[6]) {
    for (int i = 0; i < 6; ++i)
        if (hdr[i] < 0) return false;
    return hdr[0] >= 1 && hdr[1] >= 1 && hdr[4] >= 1;
}

int read_mesh_header(const char *path, int hdr[6]) {
    if (!path || !hdr) return fail(TBS_ERR_ARG, "read_mesh_header: null argument");
    FILE *fp = fopen(path, "rb");
    if (!fp) return fail(TBS_ERR_IO, std::string("could not open mesh file ") + path);
    bool ok = read_n(fp, hdr, 6);
    fclose(fp);
    if (!ok) return fail(TBS_ERR_IO, std::string("short read of mesh header in ") + path);
    if (!header_sane(hdr))
        return fail(TBS_ERR_FORMAT, std::string("invalid mesh header in ") + path);
    long long want = mesh_file_bytes(hdr), have = file_size(path);
    if (want != have)
        return fail(TBS_ERR_FORMAT, std::string("mesh file ") + path + " has " +
                                        std::to_string(have) + " bytes, header implies " +
                                        std::to_string(want));
    return TBS_OK;
}

/* one 1-based -> 0-based shift per array, read_mesh_data.F90:41-64 */
static void shift_down(int *a, size_t n) {
    for (size_t i = 0; i < n; ++i) a[i] -= 1;
}

int read_mesh(const char *path, const int hdr_in[6], int *epoint, int *ef, int *fc,
              int *linesize, int *linepoint, int *lines, int *lineface) {
    int hdr[6];
    int st = read_mesh_header(path, hdr);
    if (st) return st;
    if (hdr_in && std::memcmp(hdr, hdr_in, sizeof(hdr)) != 0)
        return fail(TBS_ERR_FORMAT, std::string("mesh header of ") + path +
                                        " differs from the sizes the caller allocated");
    if (!epoint || !ef || !fc || !linesize || !linepoint || !lines || !lineface)
        return fail(TBS_ERR_ARG, "read_mesh: null array");
    const size_t nelem = hdr[1], nint = hdr[2], eftot = hdr[3], nline = hdr[4], nle = hdr[5];
    FILE *fp = fopen(path, "rb");
    if (!fp) return fail(TBS_ERR_IO, std::string("could not open mesh file ") + path);
    int skip[6];
    bool ok = read_n(fp, skip, 6) && read_n(fp, epoint, nelem + 1) && read_n(fp, ef, eftot) &&
              read_n(fp, fc, 2 * nint) && read_n(fp, linesize, nline) &&
              read_n(fp, linepoint, nline + 1) && read_n(fp, lines, nle) &&
              read_n(fp, lineface, nle);
    fclose(fp);
    if (!ok) return fail(TBS_ERR_IO, std::string("short read of mesh arrays in ") + path);
    /* linesize is a count and keeps its value; every index array shifts */
    shift_down(epoint, nelem + 1);
    shift_down(ef, eftot);
    shift_down(fc, 2 * nint);
    shift_down(linepoint, nline + 1);
    shift_down(lines, nle);
    shift_down(lineface, nle);
    return TBS_OK;
}

int write_mesh(const char *path, const int hdr[6], const int *epoint, const int *ef,
               const int *fc, const int *linesize, const int *linepoint, const int *lines,
               const int *lineface) {
    if (!path || !hdr || !epoint || !ef || !fc || !linesize || !linepoint || !lines || !lineface)
        return fail(TBS_ERR_ARG, "write_mesh: null argument");
    if (!header_sane(hdr)) return fail(TBS_ERR_ARG, "write_mesh: invalid header");
    const size_t nelem = hdr[1], nint = hdr[2], eftot = hdr[3], nline = hdr[4], nle = hdr[5];
    FILE *fp = fopen(path, "wb");
    if (!fp) return fail(TBS_ERR_IO, std::string("could not create ") + path);
    auto put_shifted = [&](const int *a, size_t n) {
        std::vector<int> tmp(a, a + n);
        for (auto &v : tmp) v += 1;
        return write_n(fp, tmp.data(), n);
    };
    bool ok = write_n(fp, hdr, 6) && put_shifted(epoint, nelem + 1) && put_shifted(ef, eftot) &&
              put_shifted(fc, 2 * nint) && write_n(fp, linesize, nline) &&
              put_shifted(linepoint, nline + 1) && put_shifted(lines, nle) &&
              put_shifted(lineface, nle);
    ok = (fclose(fp) == 0) && ok;
    if (!ok) return fail(TBS_ERR_IO, std::string("write failed for ") + path);
    return TBS_OK;
}

int read_jacobian_header(const char *path, int hdr[3]) {
    if (!path || !hdr) return fail(TBS_ERR_ARG, "read_jacobian_header: null argument");
    FILE *fp = fopen(path, "rb");
    if (!fp) return fail(TBS_ERR_IO, std::string("could not open Jacobian file ") + path);
    bool ok = read_n(fp, hdr, 3);
    fclose(fp);
    if (!ok) return fail(TBS_ERR_IO, std::string("short read of Jacobian header in ") + path);
    if (hdr[0] < 1 || hdr[1] < 1 || hdr[2] < 0)
        return fail(TBS_ERR_FORMAT, std::string("invalid Jacobian header in ") + path);
    long long want = jacobian_file_bytes(hdr), have = file_size(path);
    if (want != have)
        return fail(TBS_ERR_FORMAT, std::string("Jacobian file ") + path + " has " +
                                        std::to_string(have) + " bytes, header implies " +
                                        std::to_string(want));
    return TBS_OK;
}

int read_jacobian(const char *path, const int hdr_in[3], double *jacD, double *jacO1,
                  double *jacO2, double *rhs, double *U0) {
    int hdr[3];
    int st = read_jacobian_header(path, hdr);
    if (st) return st;
    if (hdr_in && std::memcmp(hdr, hdr_in, sizeof(hdr)) != 0)
        return fail(TBS_ERR_FORMAT, std::string("Jacobian header of ") + path +
                                        " differs from the sizes the caller allocated");
    if (!jacD || !jacO1 || !jacO2 || !rhs || !U0)
        return fail(TBS_ERR_ARG, "read_jacobian: null array");
    const size_t nv = hdr[0], nelem = hdr[1], nint = hdr[2];
    FILE *fp = fopen(path, "rb");
    if (!fp) return fail(TBS_ERR_IO, std::string("could not open Jacobian file ") + path);
    int skip[3];
    bool ok = read_n(fp, skip, 3) && read_n(fp, jacD, nv * nv * nelem) &&
              read_n(fp, jacO1, nv * nv * nint) && read_n(fp, jacO2, nv * nv * nint) &&
              read_n(fp, rhs, nv * nelem) && read_n(fp, U0, nv * nelem);
    fclose(fp);
    if (!ok) return fail(TBS_ERR_IO, std::string("short read of Jacobian arrays in ") + path);
    return TBS_OK;
}

int write_jacobian(const char *path, const int hdr[3], const double *jacD, const double *jacO1,
                   const double *jacO2, const double *rhs, const double *U0) {
    if (!path || !hdr || !jacD || !jacO1 || !jacO2 || !rhs)
        return fail(TBS_ERR_ARG, "write_jacobian: null argument");
    if (hdr[0] < 1 || hdr[1] < 1 || hdr[2] < 0)
        return fail(TBS_ERR_ARG, "write_jacobian: invalid header");
    const size_t nv = hdr[0], nelem = hdr[1], nint = hdr[2];
    FILE *fp = fopen(path, "wb");
    if (!fp) return fail(TBS_ERR_IO, std::string("could not create ") + path);
    bool ok = write_n(fp, hdr, 3) && write_n(fp, jacD, nv * nv * nelem) &&
              write_n(fp, jacO1, nv * nv * nint) && write_n(fp, jacO2, nv * nv * nint) &&
              write_n(fp, rhs, nv * nelem);
    if (ok) {
        if (U0) {
            ok = write_n(fp, U0, nv * nelem);
        } else {
            std::vector<double> z(nv * nelem, 0.0);
            ok = write_n(fp, z.data(), z.size());
        }
    }
    ok = (fclose(fp) == 0) && ok;
    if (!ok) return fail(TBS_ERR_IO, std::string("write failed for ") + path);
    return TBS_OK;
}

int validate_mesh(const int hdr[6], const int *epoint, const int *ef, const int *fc,
                  const int *linesize, const int *linepoint, const int *lines,
                  const int *lineface) {
    if (!hdr) return fail(TBS_ERR_ARG, "validate_mesh: null header");
    if (!header_sane(hdr)) return fail(TBS_ERR_FORMAT, "mesh header has a negative or zero size");
    if (!epoint || !ef || (!fc && hdr[2] > 0) || !linesize || !linepoint || !lines || !lineface)
        return fail(TBS_ERR_ARG, "validate_mesh: null array");
    const int nelem = hdr[1], nint = hdr[2], eftot = hdr[3], nline = hdr[4], nle = hdr[5];
    if (nle != nelem)
        return fail(TBS_ERR_FORMAT, "nlineelem (" + std::to_string(nle) +
                                        ") must equal nelem (" + std::to_string(nelem) +
                                        "): every element belongs to exactly one line");
    if (epoint[0] != 0 || epoint[nelem] != eftot)
        return fail(TBS_ERR_FORMAT, "epoint must start at 0 and end at eftot");
    for (int e = 0; e < nelem; ++e)
        if (epoint[e + 1] < epoint[e])
            return fail(TBS_ERR_FORMAT, "epoint is not non-decreasing at element " + std::to_string(e));
    for (int i = 0; i < eftot; ++i)
        if (ef[i] >= nint)
            return fail(TBS_ERR_FORMAT, "ef[" + std::to_string(i) + "] = " + std::to_string(ef[i]) +
                                            " is not a face (nintface = " + std::to_string(nint) + ")");
    for (int f = 0; f < nint; ++f) {
        int a = fc[2 * f], b = fc[2 * f + 1];
        if (a < 0 || a >= nelem || b < 0 || b >= nelem || a == b)
            return fail(TBS_ERR_FORMAT, "fc of face " + std::to_string(f) + " is not a pair of distinct elements");
    }
    if (linepoint[0] != 0)
        return fail(TBS_ERR_FORMAT, "linepoint[0] must be 0");
    for (int l = 0; l < nline; ++l) {
        if (linesize[l] < 1)
            return fail(TBS_ERR_FORMAT, "line " + std::to_string(l) + " is empty");
        if (linepoint[l + 1] != linepoint[l] + linesize[l])
            return fail(TBS_ERR_FORMAT, "linepoint is not the prefix sum of linesize at line " + std::to_string(l));
    }
    if (linepoint[nline] != nle)
        return fail(TBS_ERR_FORMAT, "linepoint[nline] must equal nlineelem");
    std::vector<char> seen(nelem, 0);
    for (int m = 0; m < nle; ++m) {
        int e = lines[m];
        if (e < 0 || e >= nelem || seen[e])
            return fail(TBS_ERR_FORMAT, "lines is not a permutation of the elements (position " + std::to_string(m) + ")");
        seen[e] = 1;
    }
    for (int l = 0; l < nline; ++l) {
        for (int k = 1; k < linesize[l]; ++k) {
            int m = linepoint[l] + k;
            int f = lineface[m];
            if (f < 0 || f >= nint)
                return fail(TBS_ERR_FORMAT, "lineface[" + std::to_string(m) + "] is not an interior face");
            int a = fc[2 * f], b = fc[2 * f + 1];
            int e = lines[m], ep = lines[m - 1];
            if (!((a == e && b == ep) || (a == ep && b == e)))
                return fail(TBS_ERR_FORMAT, "lineface[" + std::to_string(m) +
                                                "] does not join consecutive line cells");
        }
    }
    return TBS_OK;
}

/* ------------------------------------------------------------ generator */

int gen_structured_header(int L, int K, int nvar, int hdr[6]) {
    if (!hdr || L < 1 || K < 1 || nvar < 1) return fail(TBS_ERR_ARG, "gen_structured_header: bad size");
    long long n = (long long)L * K;
    long long F = (long long)L * (K - 1) + (long long)(L - 1) * K;
    if (4 * n > 0x7fffffffLL) return fail(TBS_ERR_ARG, "gen_structured_header: mesh too large for int32 indices");
    hdr[0] = nvar;
    hdr[1] = (int)n;
    hdr[2] = (int)F;
    hdr[3] = (int)(4 * n);
    hdr[4] = L;
    hdr[5] = (int)n;
    return TBS_OK;
}

/* The numbering rule of the reference's ex05 data set (checked bit for bit
 * against data/ex05/gpuline.mesh.data.bin): element e = l*K + k; faces are
 * created scanning e upward, first the in-line face (e+1, e) when k+1 < K,
 * then the cross-line face (e+K, e) when l+1 < L; ef lists S, E, N, W and
 * codes boundaries as -(k+1), -(K+l+1), -(K+L+k+1), -(2K+L+l+1) on disk. */
int gen_structured_mesh(int L, int K, int *epoint, int *ef, int *fc, int *linesize,
                        int *linepoint, int *lines, int *lineface) {
    int hdr[6];
    int st = gen_structured_header(L, K, 9, hdr);
    if (st) return st;
    if (!epoint || !ef || !fc || !linesize || !linepoint || !lines || !lineface)
        return fail(TBS_ERR_ARG, "gen_structured_mesh: null array");
    const int n = hdr[1];
    std::vector<int> fidE(n, -1), fidN(n, -1);
    int nf = 0;
    for (int l = 0; l < L; ++l) {
        for (int k = 0; k < K; ++k) {
            int e = l * K + k;
            if (k + 1 < K) {
                fidE[e] = nf;
                fc[2 * nf] = e + 1;
                fc[2 * nf + 1] = e;
                ++nf;
            }
            if (l + 1 < L) {
                fidN[e] = nf;
                fc[2 * nf] = e + K;
                fc[2 * nf + 1] = e;
                ++nf;
            }
        }
    }
    /* boundary codes are the on-disk (1-based) values minus one */
    for (int l = 0; l < L; ++l) {
        for (int k = 0; k < K; ++k) {
            int e = l * K + k;
            int *row = ef + 4 * e;
            row[0] = (l > 0) ? fidN[e - K] : -(k + 1) - 1;
            row[1] = (k + 1 < K) ? fidE[e] : -(K + l + 1) - 1;
            row[2] = (l + 1 < L) ? fidN[e] : -(K + L + k + 1) - 1;
            row[3] = (k > 0) ? fidE[e - 1] : -(2 * K + L + l + 1) - 1;
            epoint[e] = 4 * e;
            lines[e] = e;
            lineface[e] = row[3];
        }
        linesize[l] = K;
        linepoint[l] = l * K;
    }
    epoint[n] = 4 * n;
    linepoint[L] = n;
    return TBS_OK;
}

static inline uint64_t splitmix64_at(uint64_t seed, uint64_t n) {
    uint64_t z = seed + (n + 1) * 0x9E3779B97F4A7C15ULL;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

static inline double uniform_pm1(uint64_t seed, uint64_t n) {
    /* 53 random bits -> [0,1) -> [-1,1); every step is exact in FP64 */
    return (double)(splitmix64_at(seed, n) >> 11) * 0x1.0p-53 * 2.0 - 1.0;
}

int gen_jacobian(int nvar, int nelem, int nintface, double shift, uint64_t seed, double *jacD,
                 double *jacO1, double *jacO2, double *rhs, double *U0) {
    if (nvar < 1 || nelem < 1 || nintface < 0)
        return fail(TBS_ERR_ARG, "gen_jacobian: bad size");
    if (!jacD || (nintface > 0 && (!jacO1 || !jacO2)) || !rhs)
        return fail(TBS_ERR_ARG, "gen_jacobian: null array");
    const long long nb = (long long)nvar * nvar;
    const long long nD = nb * nelem, nO = nb * nintface, nR = (long long)nvar * nelem;
#pragma omp parallel for schedule(static)
    for (long long i = 0; i < nD; ++i) {
        long long r = i % nvar, c = (i / nvar) % nvar;
        double u = uniform_pm1(seed, (uint64_t)i);
        jacD[i] = (r == c) ? u + shift : u;
    }
#pragma omp parallel for schedule(static)
    for (long long i = 0; i < nO; ++i) jacO1[i] = 0.1 * uniform_pm1(seed, (uint64_t)(nD + i));
#pragma omp parallel for schedule(static)
    for (long long i = 0; i < nO; ++i) jacO2[i] = 0.1 * uniform_pm1(seed, (uint64_t)(nD + nO + i));
#pragma omp parallel for schedule(static)
    for (long long i = 0; i < nR; ++i) rhs[i] = uniform_pm1(seed, (uint64_t)(nD + 2 * nO + i));
    if (U0) {
#pragma omp parallel for schedule(static)
        for (long long i = 0; i < nR; ++i) U0[i] = 0.0;
    }
    return TBS_OK;
}

}  // namespace tbs

/* =========================================================== C entry points */
using namespace tbs;

extern "C" {

void read_mesh_data_(int *nvar, int *nelem, int *nintface, int *eftot, int *nline,
                     int *nlineelem, int *epoint, int *ef, int *fc, int *lines, int *linesize,
                     int *linepoint, int *lineface) {
    if (!nvar || !nelem || !nintface || !eftot || !nline || !nlineelem) {
        set_thread_error("read_mesh_data_: null size argument");
        return;
    }
    int hdr[6] = {*nvar, *nelem, *nintface, *eftot, *nline, *nlineelem};
    read_mesh("gpuline.mesh.data.bin", hdr, epoint, ef, fc, linesize, linepoint, lines, lineface);
}

void read_jacobian_data_(int *nvar, int *nelem, int *nintface, double *jacD, double *jacO1,
                         double *jacO2, double *rhs, double *U0) {
    if (!nvar || !nelem || !nintface) {
        set_thread_error("read_jacobian_data_: null size argument");
        return;
    }
    int hdr[3] = {*nvar, *nelem, *nintface};
    read_jacobian("gpuline.jacobian.data.bin", hdr, jacD, jacO1, jacO2, rhs, U0);
}

int tbs_read_mesh_header(const char *path, int hdr[6]) { return read_mesh_header(path, hdr); }

int tbs_read_mesh(const char *path, const int hdr[6], int *epoint, int *ef, int *fc, int *linesize,
                  int *linepoint, int *lines, int *lineface) {
    return read_mesh(path, hdr, epoint, ef, fc, linesize, linepoint, lines, lineface);
}

int tbs_write_mesh(const char *path, const int hdr[6], const int *epoint, const int *ef,
                   const int *fc, const int *linesize, const int *linepoint, const int *lines,
                   const int *lineface) {
    return write_mesh(path, hdr, epoint, ef, fc, linesize, linepoint, lines, lineface);
}

int tbs_read_jacobian_header(const char *path, int hdr[3]) { return read_jacobian_header(path, hdr); }

int tbs_read_jacobian(const char *path, const int hdr[3], double *jacD, double *jacO1,
                      double *jacO2, double *rhs, double *U0) {
    return read_jacobian(path, hdr, jacD, jacO1, jacO2, rhs, U0);
}

int tbs_write_jacobian(const char *path, const int hdr[3], const double *jacD,
                       const double *jacO1, const double *jacO2, const double *rhs,
                       const double *U0) {
    return write_jacobian(path, hdr, jacD, jacO1, jacO2, rhs, U0);
}

int tbs_validate_mesh(const int hdr[6], const int *epoint, const int *ef, const int *fc,
                      const int *linesize, const int *linepoint, const int *lines,
                      const int *lineface) {
    return validate_mesh(hdr, epoint, ef, fc, linesize, linepoint, lines, lineface);
}

int tbs_gen_structured_header(int L, int K, int nvar, int hdr[6]) {
    return gen_structured_header(L, K, nvar, hdr);
}

int tbs_gen_structured_mesh(int L, int K, int *epoint, int *ef, int *fc, int *linesize,
                            int *linepoint, int *lines, int *lineface) {
    return gen_structured_mesh(L, K, epoint, ef, fc, linesize, linepoint, lines, lineface);
}

int tbs_gen_jacobian(int nvar, int nelem, int nintface, double shift, uint64_t seed, double *jacD,
                     double *jacO1, double *jacO2, double *rhs, double *U0) {
    return gen_jacobian(nvar, nelem, nintface, shift, seed, jacD, jacO1, jacO2, rhs, U0);
}

int tbs_resize_block_size(int nv_old, int nv_new, int nelem, int nintface, const double *D_old,
                          const double *O1_old, const double *O2_old, const double *rhs_old,
                          const double *U0_old, double *D, double *O1, double *O2, double *rhs,
                          double *U0) {
    if (nv_old < 1 || nv_new < 1 || nelem < 1 || nintface < 0)
        return fail(TBS_ERR_ARG, "tbs_resize_block_size: bad size");
    if (!D_old || !rhs_old || !U0_old || !D || !rhs || !U0 ||
        (nintface > 0 && (!O1_old || !O2_old || !O1 || !O2)))
        return fail(TBS_ERR_ARG, "tbs_resize_block_size: null array");
    const size_t bo = (size_t)nv_old * nv_old, bn = (size_t)nv_new * nv_new;
    const int mn = nv_new < nv_old ? nv_new : nv_old;
    /* std::vector::resize keeps the leading old entries, zero-fills the rest */
    auto keep = [](const double *src, size_t nsrc, double *dst, size_t ndst) {
        for (size_t i = 0; i < ndst; ++i) dst[i] = i < nsrc ? src[i] : 0.0;
    };
    keep(D_old, bo * nelem, D, bn * nelem);
    keep(O1_old, bo * nintface, O1, bn * nintface);
    keep(O2_old, bo * nintface, O2, bn * nintface);
    keep(rhs_old, (size_t)nv_old * nelem, rhs, (size_t)nv_new * nelem);
    keep(U0_old, (size_t)nv_old * nelem, U0, (size_t)nv_new * nelem);
    for (int e = 0; e < nelem; ++e)
        for (int j = 0; j < nv_new; ++j) D[e * bn + (size_t)nv_new * j + j] = 10.0;
    for (int f = 0; f < nintface; ++f)
        for (int j = 0; j < nv_new; ++j) {
            O1[f * bn + (size_t)nv_new * j + j] = 10.0;
            O2[f * bn + (size_t)nv_new * j + j] = 10.0;
        }
    for (int e = 0; e < nelem; ++e)
        for (int j = 0; j < mn; ++j)
            for (int i = 0; i < mn; ++i)
                D[e * bn + (size_t)nv_new * j + i] = D_old[e * bo + (size_t)nv_old * j + i];
    for (int f = 0; f < nintface; ++f)
        for (int j = 0; j < mn; ++j)
            for (int i = 0; i < mn; ++i) {
                O1[f * bn + (size_t)nv_new * j + i] = O1_old[f * bo + (size_t)nv_old * j + i];
                O2[f * bn + (size_t)nv_new * j + i] = O2_old[f * bo + (size_t)nv_old * j + i];
            }
    for (size_t eij = 0; eij < (size_t)nelem * mn; ++eij) {
        rhs[eij] = rhs_old[eij];
        U0[eij] = U0_old[eij];
    }
    return TBS_OK;
}

const char *tbs_version(void) { return "triblocksolve_b200 0.1.0 (sm_100a)"; }

}  // extern "C"
