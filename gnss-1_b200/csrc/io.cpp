// io.cpp -- the reference's file formats (iofuncs.cu) and an exact checkpoint,
// on the C ABI of gnss_b200.h.
//
// Reference formats (all native-endian doubles, as fwrite writes them):
//   3D field   double(8 nx ny nz), then f[x][y][z] for z fastest   (write3Dfields_mgpu, iofuncs.cu:329-358)
//   xy plane   double(8 nx ny), then f[x][y][z0]                    (writexyfields, iofuncs.cu:187-209)
//   xz plane   double(8 nx nz), then f[x][y0][z]                    (writexzfields, iofuncs.cu:211-233)
//   yz plane   double(8 ny nz), then f[x0][y][z]                    (writeyzfields, iofuncs.cu:235-257)
//   statistic  one double per record, appended                      (writeStats, iofuncs.cu:128-146)
//   profile    ny doubles                                           (writeYprofs, iofuncs.cu:78-98)
// Host arrays use the reference's padded in-place layout [nx][ny][2 (nz/2+1)].
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "gnss_b200.h"

namespace {

struct File {
    FILE *f = nullptr;
    File(const char *path, const char *mode) : f(std::fopen(path, mode)) {}
    ~File() {
        if (f) std::fclose(f);
    }
};

bool dims_ok(int nx, int ny, int nz) { return nx > 0 && ny > 0 && nz > 0 && nz % 2 == 0; }
size_t pidx(int ny, int nz, int i, int j, int k) { return (size_t)k + 2 * (size_t)(nz / 2 + 1) * (j + (size_t)ny * i); }

gnss_status write_doubles(FILE *f, const double *v, size_t n) {
    return std::fwrite(v, sizeof(double), n, f) == n ? GNSS_OK : GNSS_ERR_INVALID;
}

}  // namespace

gnss_status gnss_io_write_field(int nx, int ny, int nz, const double *phys, const char *path) {
    if (!dims_ok(nx, ny, nz) || !phys || !path) return GNSS_ERR_INVALID;
    File out(path, "wb");
    if (!out.f) return GNSS_ERR_INVALID;
    const double bytes = (double)(sizeof(double) * (size_t)nx * ny * nz);
    if (write_doubles(out.f, &bytes, 1)) return GNSS_ERR_INVALID;
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j)
            if (write_doubles(out.f, phys + pidx(ny, nz, i, j, 0), (size_t)nz)) return GNSS_ERR_INVALID;
    return GNSS_OK;
}

gnss_status gnss_io_read_field(int nx, int ny, int nz, const char *path, double *phys) {
    if (!dims_ok(nx, ny, nz) || !phys || !path) return GNSS_ERR_INVALID;
    File in(path, "rb");
    if (!in.f) return GNSS_ERR_INVALID;
    double bytes = 0.0;
    if (std::fread(&bytes, sizeof(double), 1, in.f) != 1) return GNSS_ERR_INVALID;
    if (bytes / sizeof(double) != (double)nx * ny * nz) return GNSS_ERR_INVALID;   // iofuncs.cu:472-476
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j)
            if (std::fread(phys + pidx(ny, nz, i, j, 0), sizeof(double), (size_t)nz, in.f) != (size_t)nz)
                return GNSS_ERR_INVALID;
    return GNSS_OK;
}

gnss_status gnss_io_write_slice(int nx, int ny, int nz, const double *phys, int plane, int index, const char *path) {
    if (!dims_ok(nx, ny, nz) || !phys || !path) return GNSS_ERR_INVALID;
    const int lim = plane == GNSS_PLANE_XY ? nz : plane == GNSS_PLANE_XZ ? ny : plane == GNSS_PLANE_YZ ? nx : -1;
    if (lim < 0 || index < 0 || index >= lim) return GNSS_ERR_INVALID;
    File out(path, "wb");
    if (!out.f) return GNSS_ERR_INVALID;
    std::vector<double> v;
    if (plane == GNSS_PLANE_XY) {
        v.push_back((double)(sizeof(double) * (size_t)nx * ny));
        for (int i = 0; i < nx; ++i)
            for (int j = 0; j < ny; ++j) v.push_back(phys[pidx(ny, nz, i, j, index)]);
    } else if (plane == GNSS_PLANE_XZ) {
        v.push_back((double)(sizeof(double) * (size_t)nx * nz));
        for (int i = 0; i < nx; ++i)
            for (int k = 0; k < nz; ++k) v.push_back(phys[pidx(ny, nz, i, index, k)]);
    } else {
        v.push_back((double)(sizeof(double) * (size_t)ny * nz));
        for (int j = 0; j < ny; ++j)
            for (int k = 0; k < nz; ++k) v.push_back(phys[pidx(ny, nz, index, j, k)]);
    }
    return write_doubles(out.f, v.data(), v.size());
}

gnss_status gnss_io_write_stat(const char *path, double value, int append) {
    if (!path) return GNSS_ERR_INVALID;
    File out(path, append ? "ab" : "wb");
    if (!out.f) return GNSS_ERR_INVALID;
    return write_doubles(out.f, &value, 1);
}

gnss_status gnss_io_write_profile(int ny, const double *prof, const char *path) {
    if (ny <= 0 || !prof || !path) return GNSS_ERR_INVALID;
    File out(path, "wb");
    if (!out.f) return GNSS_ERR_INVALID;
    return write_doubles(out.f, prof, (size_t)ny);
}

// ------------------------------------------------------------------ device states
namespace {

struct Dev {
    void *p = nullptr;
    ~Dev() {
        if (p) cudaFree(p);
    }
};

void field_ptrs(const gnss_fields *f, void *out[5]) {
    out[0] = f->u;
    out[1] = f->v;
    out[2] = f->w;
    out[3] = f->s;
    out[4] = f->c;
}

const char kVar[5] = {'u', 'v', 'w', 'z', 'c'};   // save3Dfields' file names (iofuncs.cu:391-395)

std::string var_path(const char *dir, int q, int iter) {
    return std::string(dir) + "/" + kVar[q] + "." + std::to_string(iter);
}

}  // namespace

gnss_status gnss_save_state(gnss_ctx *ctx, const gnss_fields *state, const char *dir, int iter, void *stream) {
    gnss_config cfg;
    if (!ctx || !state || !dir || gnss_get_config(ctx, &cfg)) return GNSS_ERR_INVALID;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    const size_t fb = gnss_field_bytes(ctx);
    const size_t nreal = fb / (cfg.precision == GNSS_FP64 ? 8 : 4);   // padded real values
    Dev tmp;
    if (cudaSetDevice(cfg.device) != cudaSuccess || cudaMalloc(&tmp.p, fb) != cudaSuccess) {
        cudaGetLastError();
        return GNSS_ERR_NOMEM;
    }
    std::vector<unsigned char> raw(fb);
    std::vector<double> phys(nreal, 0.0);
    void *f[5];
    field_ptrs(state, f);
    for (int q = 0; q < 5; ++q) {
        if (q >= 3 + cfg.n_scalars && q != 4) continue;
        if (f[q]) {
            if (cudaMemcpyAsync(tmp.p, f[q], fb, cudaMemcpyDeviceToDevice, s) != cudaSuccess) return GNSS_ERR_CUDA;
            gnss_status st = gnss_inverse(ctx, tmp.p, stream);
            if (st) return st;
            if (cudaMemcpyAsync(raw.data(), tmp.p, fb, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
                cudaStreamSynchronize(s) != cudaSuccess)
                return GNSS_ERR_CUDA;
            if (cfg.precision == GNSS_FP64) {
                std::memcpy(phys.data(), raw.data(), fb);
            } else {
                const float *r = reinterpret_cast<const float *>(raw.data());
                for (size_t i = 0; i < nreal; ++i) phys[i] = r[i];
            }
        } else {
            std::fill(phys.begin(), phys.end(), 0.0);   // the reference always writes c
        }
        gnss_status st = gnss_io_write_field(cfg.nx, cfg.ny, cfg.nz, phys.data(), var_path(dir, q, iter).c_str());
        if (st) return st;
    }
    return GNSS_OK;
}

gnss_status gnss_load_state(gnss_ctx *ctx, const char *dir, int iter, const gnss_fields *state, void *stream) {
    gnss_config cfg;
    if (!ctx || !state || !dir || gnss_get_config(ctx, &cfg)) return GNSS_ERR_INVALID;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    const size_t fb = gnss_field_bytes(ctx);
    const size_t nreal = fb / (cfg.precision == GNSS_FP64 ? 8 : 4);
    if (cudaSetDevice(cfg.device) != cudaSuccess) return GNSS_ERR_CUDA;
    std::vector<double> phys(nreal);
    std::vector<float> phys32(cfg.precision == GNSS_FP32 ? nreal : 0);
    void *f[5];
    field_ptrs(state, f);
    const int nf = 3 + cfg.n_scalars;
    for (int q = 0; q < nf; ++q) {
        if (!f[q]) return GNSS_ERR_INVALID;
        std::fill(phys.begin(), phys.end(), 0.0);
        gnss_status st = gnss_io_read_field(cfg.nx, cfg.ny, cfg.nz, var_path(dir, q, iter).c_str(), phys.data());
        if (st && q < 3) return st;          // the velocity must be there; a missing scalar stays zero
        if (st) std::fill(phys.begin(), phys.end(), 0.0);
        const void *src = phys.data();
        if (cfg.precision == GNSS_FP32) {
            for (size_t i = 0; i < nreal; ++i) phys32[i] = (float)phys[i];
            src = phys32.data();
        }
        if (cudaMemcpyAsync(f[q], src, fb, cudaMemcpyHostToDevice, s) != cudaSuccess) return GNSS_ERR_CUDA;
        if ((st = gnss_forward(ctx, f[q], stream))) return st;
        if (cudaStreamSynchronize(s) != cudaSuccess) return GNSS_ERR_CUDA;   // host buffers are reused
    }
    return GNSS_OK;
}

// ------------------------------------------------------------------ checkpoint
namespace {

const char kMagic[8] = {'G', 'N', 'S', 'S', 'C', 'K', 'P', '1'};

struct CkptHeader {
    char magic[8];
    int32_t nx, ny, nz, precision, n_scalars, scheme, nfields, has_hist;
    int64_t step;
    uint64_t field_bytes;
};

}  // namespace

gnss_status gnss_checkpoint_save(gnss_ctx *ctx, const gnss_fields *state, const gnss_fields *hist, long long step,
                                 const char *path, void *stream) {
    gnss_config cfg;
    if (!ctx || !state || !path || gnss_get_config(ctx, &cfg)) return GNSS_ERR_INVALID;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    const size_t fb = gnss_field_bytes(ctx);
    const int nf = 3 + cfg.n_scalars;
    CkptHeader h{};
    std::memcpy(h.magic, kMagic, 8);
    h.nx = cfg.nx;
    h.ny = cfg.ny;
    h.nz = cfg.nz;
    h.precision = cfg.precision;
    h.n_scalars = cfg.n_scalars;
    h.scheme = cfg.scheme;
    h.nfields = nf;
    h.has_hist = hist ? 1 : 0;
    h.step = step;
    h.field_bytes = fb;
    if (cudaSetDevice(cfg.device) != cudaSuccess) return GNSS_ERR_CUDA;
    File out(path, "wb");
    if (!out.f || std::fwrite(&h, sizeof h, 1, out.f) != 1) return GNSS_ERR_INVALID;
    std::vector<unsigned char> raw(fb);
    for (int set = 0; set < 1 + h.has_hist; ++set) {
        void *f[5];
        field_ptrs(set == 0 ? state : hist, f);
        for (int q = 0; q < nf; ++q) {
            if (!f[q]) return GNSS_ERR_INVALID;
            if (cudaMemcpyAsync(raw.data(), f[q], fb, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
                cudaStreamSynchronize(s) != cudaSuccess)
                return GNSS_ERR_CUDA;
            if (std::fwrite(raw.data(), 1, fb, out.f) != fb) return GNSS_ERR_INVALID;
        }
    }
    return GNSS_OK;
}

gnss_status gnss_checkpoint_load(gnss_ctx *ctx, const char *path, const gnss_fields *state, const gnss_fields *hist,
                                 long long *step, void *stream) {
    gnss_config cfg;
    if (!ctx || !state || !path || gnss_get_config(ctx, &cfg)) return GNSS_ERR_INVALID;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    const size_t fb = gnss_field_bytes(ctx);
    const int nf = 3 + cfg.n_scalars;
    File in(path, "rb");
    CkptHeader h{};
    if (!in.f || std::fread(&h, sizeof h, 1, in.f) != 1 || std::memcmp(h.magic, kMagic, 8) != 0) return GNSS_ERR_INVALID;
    if (h.nx != cfg.nx || h.ny != cfg.ny || h.nz != cfg.nz || h.precision != cfg.precision ||
        h.n_scalars != cfg.n_scalars || h.scheme != cfg.scheme || h.nfields != nf || h.field_bytes != fb ||
        (hist && !h.has_hist))
        return GNSS_ERR_INVALID;
    if (cudaSetDevice(cfg.device) != cudaSuccess) return GNSS_ERR_CUDA;
    std::vector<unsigned char> raw(fb);
    for (int set = 0; set < 1 + h.has_hist; ++set) {
        void *f[5];
        if (set == 1 && !hist) break;
        field_ptrs(set == 0 ? state : hist, f);
        for (int q = 0; q < nf; ++q) {
            if (!f[q] || std::fread(raw.data(), 1, fb, in.f) != fb) return GNSS_ERR_INVALID;
            if (cudaMemcpyAsync(f[q], raw.data(), fb, cudaMemcpyHostToDevice, s) != cudaSuccess ||
                cudaStreamSynchronize(s) != cudaSuccess)
                return GNSS_ERR_CUDA;
        }
    }
    if (step) *step = h.step;
    return GNSS_OK;
}
