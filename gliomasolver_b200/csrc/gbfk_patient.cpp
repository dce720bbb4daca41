// Patient data for the RD path: the reference's Matrix files and the mapping
// of GM/WM/CSF volumes plus the tumour initial condition onto the grid
// (Glioma_ReactionDiffusion::_ic, Glioma/Glioma_ReactionDiffusion.cpp:79-172).
//
// Host code: the mapping runs once per anatomy (a TMCMC stage shares it),
// so it stays on the CPU, spread over host threads by z-plane.  Its
// arithmetic is the reference's, in the reference's Real, including the
// float/double mix of the default float build; glibc's sin and the IEEE
// division and square root give the same bits as the reference's cells.
#include "gbfk.h"
#include "gbfk_host.h"

#include <algorithm>
#include <cerrno>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

namespace {

thread_local std::string g_host_err;

int host_fail(int code, const char *fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_host_err = buf;
    return code;
}

struct File {
    FILE *f = nullptr;
    ~File()
    {
        if (f) fclose(f);
    }
};

// Matrix.h:20-34 (layout), :71-88 (deserializeHeader), :141-169 (type id).
int read_header(FILE *f, const char *path, int *dim, int sizes[3], int *type_id)
{
    int32_t h[2];
    if (fread(h, sizeof(int32_t), 2, f) != 2) return host_fail(GBFK_E_IO, "%s: short header", path);
    if (h[0] != 1234) return host_fail(GBFK_E_IO, "%s: magic number %d, not 1234", path, (int)h[0]);
    if (h[1] != 2 && h[1] != 3) return host_fail(GBFK_E_IO, "%s: dimension %d, not 2 or 3", path, (int)h[1]);
    int32_t s[3] = {1, 1, 1};
    if (fread(s, sizeof(int32_t), (size_t)h[1], f) != (size_t)h[1])
        return host_fail(GBFK_E_IO, "%s: short header", path);
    for (int d = 0; d < h[1]; d++)
        if (s[d] < 0) return host_fail(GBFK_E_IO, "%s: negative size %d", path, (int)s[d]);
    int32_t t;
    if (fread(&t, sizeof(int32_t), 1, f) != 1) return host_fail(GBFK_E_IO, "%s: missing type id", path);
    if (t < 0 || t > 2) return host_fail(GBFK_E_IO, "%s: unknown type id %d", path, (int)t);
    *dim = h[1];
    for (int d = 0; d < 3; d++) sizes[d] = s[d];
    *type_id = t;
    return GBFK_OK;
}

template <class T>
int read_values(FILE *f, const char *path, double *out, int64_t n)
{
    const int64_t chunk = 1 << 16;
    std::vector<T> tmp((size_t)std::min<int64_t>(n, chunk));
    for (int64_t i = 0; i < n; i += chunk) {
        const int64_t m = std::min<int64_t>(chunk, n - i);
        if (fread(tmp.data(), sizeof(T), (size_t)m, f) != (size_t)m)
            return host_fail(GBFK_E_IO, "%s: short data (%lld of %lld values)", path, (long long)i, (long long)n);
        for (int64_t j = 0; j < m; j++) out[i + j] = (double)tmp[(size_t)j];
    }
    return GBFK_OK;
}

template <class T>
int write_values(FILE *f, const char *path, const double *data, int64_t n)
{
    const int64_t chunk = 1 << 16;
    std::vector<T> tmp((size_t)std::min<int64_t>(n, chunk));
    for (int64_t i = 0; i < n; i += chunk) {
        const int64_t m = std::min<int64_t>(chunk, n - i);
        for (int64_t j = 0; j < m; j++) tmp[(size_t)j] = (T)data[i + j];
        if (fwrite(tmp.data(), sizeof(T), (size_t)m, f) != (size_t)m)
            return host_fail(GBFK_E_IO, "%s: write failed", path);
    }
    return GBFK_OK;
}

struct MapArgs {
    int ncell;          // cells per direction (8 * bpd)
    double inv_extent;  // 1 / (8 * 2^level): cell spacing of the grid
    int msize[3];
    int mmax;
    const double *gm, *wm, *csf;
    double tic[3];
    void *pw, *pg, *pcsf, *phi, *tissue;
};

// The tumour profile of _ic at one cell (:155-164), in Real: 0 = the ball's
// core (psi < -1), 1 = the smoothing band (-1 <= psi <= 1; *value is the
// profile there), 2 = outside (also for a NaN psi, as the reference's
// comparisons then all fail).
template <class Real>
inline int ball_zone(const Real x[3], const Real tic[3], Real *value)
{
    // :103-106: tumour radius, smoothing support and width (fixed h = 1/128)
    const Real tumorRadius = (Real)0.005;
    const Real smooth_sup = (Real)2.;
    const Real h = (Real)(1. / 128);
    const Real iw = (Real)(1. / (smooth_sup * h));
    const Real p[3] = {(Real)(x[0] - tic[0]), (Real)(x[1] - tic[1]), (Real)(x[2] - tic[2])};
    const Real dist = std::sqrt((Real)((Real)(p[0] * p[0]) + (Real)(p[1] * p[1])) + (Real)(p[2] * p[2]));
    const Real psi = (Real)((Real)(dist - tumorRadius) * iw);
    if (psi < (Real)-1) return 0;
    if ((Real)-1 <= psi && psi <= (Real)1) {
        *value = (Real)(1.0 * 0.5 * ((double)(Real)((Real)1 - psi) - sin(M_PI * (double)psi) / (M_PI)));
        return 1;
    }
    return 2;
}

// BlockInfo::pos of grid cell i: origin + h * i, exact multiples of the spacing.
template <class Real>
inline Real cell_pos(int i, double spacing)
{
    return (Real)(i * spacing);
}

inline double grid_spacing(int bpd)
{
    // MRAG places bpd blocks at level ceil(log2 bpd) (MRAGridHelpers.h:9-17),
    // block spacing 2^-level (MRAGrid.inl:200-212).
    int level = 0;
    while ((1 << level) < bpd) level++;
    return 1.0 / (double)(8 << level);
}

// One z-plane range of Glioma_ReactionDiffusion::_ic (:117-167), in Real.
template <class Real>
void map_planes(const MapArgs &a, int z0, int z1)
{
    const int n = a.ncell;
    // :98-100: voxel spacing w.r.t. the longest dimension
    const double brainH = 1.0 / (double)a.mmax;
    const Real tic[3] = {(Real)a.tic[0], (Real)a.tic[1], (Real)a.tic[2]};
    Real *o_pw = (Real *)a.pw, *o_pg = (Real *)a.pg, *o_csf = (Real *)a.pcsf;
    Real *o_phi = (Real *)a.phi, *o_t = (Real *)a.tissue;
    const int64_t sx = a.msize[0], sy = a.msize[1], sz = a.msize[2];

    for (int iz = z0; iz < z1; iz++)
        for (int iy = 0; iy < n; iy++)
            for (int ix = 0; ix < n; ix++) {
                const int64_t c = ix + (int64_t)n * (iy + (int64_t)n * iz);
                const Real x[3] = {cell_pos<Real>(ix, a.inv_extent), cell_pos<Real>(iy, a.inv_extent),
                                   cell_pos<Real>(iz, a.inv_extent)};
                const int mx = (int)floor((double)x[0] / brainH);
                const int my = (int)floor((double)x[1] / brainH);
                const int mz = (int)floor((double)x[2] / brainH);
                Real w = 0, g = 0, f = 0, ph = 0, t = 0;
                if ((mx >= 0 && mx < sx) & (my >= 0 && my < sy) && (mz >= 0 && mz < sz)) {
                    const int64_t v = mx + sx * (my + sy * (int64_t)mz);
                    Real pGM = (Real)a.gm[v], pWM = (Real)a.wm[v], pCSF = (Real)a.csf[v];
                    // :144-147: the vote compares with the already replaced pCSF
                    double tissue = (double)(Real)(pWM + pGM);
                    pCSF = ((double)pCSF > tissue) ? (Real)1. : (Real)0.;
                    pWM = ((double)pCSF > tissue) ? (Real)0. : pWM;
                    pGM = ((double)pCSF > tissue) ? (Real)0. : pGM;
                    // :149-152
                    tissue = (double)(Real)(pWM + pGM);
                    w = (tissue > 0.) ? (Real)((double)pWM / tissue) : (Real)0.;
                    g = (tissue > 0.) ? (Real)((double)pGM / tissue) : (Real)0.;
                    f = pCSF;
                    t = (Real)(pGM + pWM);
                    // :157-164
                    Real band = 0;
                    const int zone = ball_zone<Real>(x, tic, &band);
                    if (zone == 0 && (double)t > 0.001)
                        ph = (Real)1.0;
                    else if (zone == 1 && (double)t > 0)
                        ph = band;
                    else
                        ph = (Real)0.0;
                }
                if (o_pw) o_pw[c] = w;
                if (o_pg) o_pg[c] = g;
                if (o_csf) o_csf[c] = f;
                if (o_phi) o_phi[c] = ph;
                if (o_t) o_t[c] = t;
            }
}

template <class Real>
void map_all(const MapArgs &a)
{
    const int n = a.ncell;
    unsigned hw = std::thread::hardware_concurrency();
    int nt = (int)std::max(1u, std::min<unsigned>(hw ? hw : 1u, 64u));
    nt = std::min(nt, n);
    if (nt <= 1) {
        map_planes<Real>(a, 0, n);
        return;
    }
    std::vector<std::thread> th;
    for (int k = 0; k < nt; k++) {
        const int z0 = (int)((int64_t)n * k / nt), z1 = (int)((int64_t)n * (k + 1) / nt);
        th.emplace_back([&a, z0, z1] { map_planes<Real>(a, z0, z1); });
    }
    for (auto &t : th) t.join();
}

}  // namespace

namespace gbfk_host {

template <class Real>
bool ball_band_cells(int bpd, const double tic_d[3], std::vector<BallCell<Real>> &out)
{
    out.clear();
    const int n = 8 * bpd;
    const double sp = grid_spacing(bpd);
    const Real tic[3] = {(Real)tic_d[0], (Real)tic_d[1], (Real)tic_d[2]};
    // the band ends at radius 0.005 + 1/64; two cells of margin cover the
    // rounding of the distance in Real
    const double reach = 0.005 + 1. / 64;
    int lo[3], hi[3];
    for (int d = 0; d < 3; d++) {
        const double c = (double)tic[d];
        if (!(c == c)) return true;  // NaN centre: every cell is outside
        const double l = std::floor((c - reach) / sp) - 2, u = std::ceil((c + reach) / sp) + 2;
        lo[d] = (int)std::max(0.0, std::min((double)n, l));
        hi[d] = (int)std::max(-1.0, std::min((double)(n - 1), u));
    }
    for (int iz = lo[2]; iz <= hi[2]; iz++)
        for (int iy = lo[1]; iy <= hi[1]; iy++)
            for (int ix = lo[0]; ix <= hi[0]; ix++) {
                const Real x[3] = {cell_pos<Real>(ix, sp), cell_pos<Real>(iy, sp), cell_pos<Real>(iz, sp)};
                Real v = 0;
                const int zone = ball_zone<Real>(x, tic, &v);
                if (zone == 0) return false;
                if (zone == 1) out.push_back(BallCell<Real>{ix, iy, iz, v});
            }
    return true;
}

template bool ball_band_cells<float>(int, const double[3], std::vector<BallCell<float>> &);
template bool ball_band_cells<double>(int, const double[3], std::vector<BallCell<double>> &);

}  // namespace gbfk_host

extern "C" {

const char *gbfk_host_last_error(void) { return g_host_err.c_str(); }

int gbfk_matrix_info(const char *path, int *dim, int sizes[3], int *type_id)
{
    if (!path || !dim || !sizes || !type_id) return host_fail(GBFK_E_INVALID, "gbfk_matrix_info: NULL argument");
    File f;
    f.f = fopen(path, "rb");
    if (!f.f) return host_fail(GBFK_E_IO, "%s: cannot open: %s", path, strerror(errno));
    return read_header(f.f, path, dim, sizes, type_id);
}

int gbfk_matrix_read(const char *path, double *out, int64_t capacity)
{
    if (!path || (!out && capacity > 0)) return host_fail(GBFK_E_INVALID, "gbfk_matrix_read: NULL argument");
    File f;
    f.f = fopen(path, "rb");
    if (!f.f) return host_fail(GBFK_E_IO, "%s: cannot open: %s", path, strerror(errno));
    int dim, sizes[3], tid;
    int rc = read_header(f.f, path, &dim, sizes, &tid);
    if (rc) return rc;
    const int64_t n = (int64_t)sizes[0] * sizes[1] * sizes[2];
    if (n > capacity)
        return host_fail(GBFK_E_INVALID, "%s: %lld values, capacity %lld", path, (long long)n, (long long)capacity);
    switch (tid) {
    case 0: return read_values<double>(f.f, path, out, n);
    case 1: return read_values<float>(f.f, path, out, n);
    default: return read_values<int32_t>(f.f, path, out, n);
    }
}

int gbfk_matrix_write(const char *path, int dim, const int *sizes, int type_id, const double *data)
{
    if (!path || !sizes || (dim != 2 && dim != 3) || type_id < 0 || type_id > 2)
        return host_fail(GBFK_E_INVALID, "gbfk_matrix_write: bad arguments");
    int64_t n = 1;
    for (int d = 0; d < dim; d++) {
        if (sizes[d] < 0) return host_fail(GBFK_E_INVALID, "gbfk_matrix_write: negative size");
        n *= sizes[d];
    }
    if (n > 0 && !data) return host_fail(GBFK_E_INVALID, "gbfk_matrix_write: NULL data");
    if (type_id == 2)
        for (int64_t i = 0; i < n; i++)
            if (!(data[i] > -2147483649.0 && data[i] < 2147483648.0))
                return host_fail(GBFK_E_INVALID, "gbfk_matrix_write: value %g at %lld is not an int32", data[i],
                                 (long long)i);
    File f;
    f.f = fopen(path, "wb");
    if (!f.f) return host_fail(GBFK_E_IO, "%s: cannot create: %s", path, strerror(errno));
    int32_t head[5] = {1234, dim, sizes[0], sizes[1], dim == 3 ? sizes[2] : 0};
    int32_t tid = type_id;
    if (fwrite(head, sizeof(int32_t), (size_t)(2 + dim), f.f) != (size_t)(2 + dim) ||
        fwrite(&tid, sizeof(int32_t), 1, f.f) != 1)
        return host_fail(GBFK_E_IO, "%s: write failed", path);
    int rc;
    switch (type_id) {
    case 0: rc = write_values<double>(f.f, path, data, n); break;
    case 1: rc = write_values<float>(f.f, path, data, n); break;
    default: rc = write_values<int32_t>(f.f, path, data, n); break;
    }
    if (rc) return rc;
    FILE *ff = f.f;
    f.f = nullptr;
    if (fclose(ff) != 0) return host_fail(GBFK_E_IO, "%s: close failed", path);
    return GBFK_OK;
}

int gbfk_map_anatomy(int precision, int bpd, const int msize[3], const double *gm, const double *wm,
                     const double *csf, const double tumor_ic[3], void *pw, void *pg, void *pcsf, void *phi,
                     void *tissue, double *L)
{
    if (precision != GBFK_F64 && precision != GBFK_F32)
        return host_fail(GBFK_E_INVALID, "gbfk_map_anatomy: precision %d", precision);
    if (bpd < 1 || bpd > 4096) return host_fail(GBFK_E_INVALID, "gbfk_map_anatomy: bpd %d", bpd);
    if (!msize || !gm || !wm || !csf || !tumor_ic)
        return host_fail(GBFK_E_INVALID, "gbfk_map_anatomy: NULL argument");
    MapArgs a;
    a.mmax = 0;
    for (int d = 0; d < 3; d++) {
        if (msize[d] < 1) return host_fail(GBFK_E_INVALID, "gbfk_map_anatomy: volume size %d", msize[d]);
        a.msize[d] = msize[d];
        a.mmax = std::max(a.mmax, msize[d]);
        a.tic[d] = tumor_ic[d];
    }
    a.ncell = 8 * bpd;
    a.inv_extent = grid_spacing(bpd);
    a.gm = gm;
    a.wm = wm;
    a.csf = csf;
    a.pw = pw;
    a.pg = pg;
    a.pcsf = pcsf;
    a.phi = phi;
    a.tissue = tissue;
    // :96: L = brainSizeMax * 0.1, stored in Real
    if (precision == GBFK_F64) {
        map_all<double>(a);
        if (L) *L = (double)a.mmax * 0.1;
    } else {
        map_all<float>(a);
        if (L) *L = (double)(float)((double)a.mmax * 0.1);
    }
    return GBFK_OK;
}

}  // extern "C"
