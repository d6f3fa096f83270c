// C ABI of sonium-b200 (declared in include/sonium_b200.h). Every entry point catches
// failures and turns them into a status code plus a thread-local message; nothing falls back
// to a CPU computation.

#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>

#include "sb_blas.cuh"
#include "sb_internal.cuh"
#include "sb_profile.cuh"

struct sb_mesh {
    sb::Mesh* m;
};
struct sb_operator {
    sb::Operator* op;
};
struct sb_gcro_subspace {
    sb::RecycleSpace* s;
};

namespace sb {

static thread_local std::string t_err;
int g_inject_point = SB_INJECT_NONE;
static std::mutex g_inject_mu;

void set_error(int, const std::string& msg) { t_err = msg; }
void clear_error() { t_err.clear(); }

void maybe_inject(int point) {
    std::lock_guard<std::mutex> lock(g_inject_mu);
    if (g_inject_point != SB_INJECT_NONE && g_inject_point == point) {
        g_inject_point = SB_INJECT_NONE;
        throw Error{SB_ERR_INJECTED, point == SB_INJECT_ALLOC ? "injected allocation failure"
                                                              : "injected launch failure"};
    }
}

// ---- caching device allocator ----
namespace {
std::mutex g_mem_mu;
// Free blocks per (device, rounded size).
std::map<std::pair<int, size_t>, std::vector<void*>> g_free;
std::map<int, int64_t> g_in_use, g_cached;
constexpr size_t kCacheLimit = size_t(96) << 30;  // per device; larger releases go back to the driver

// SB_DEVICE_CACHE=0 in the environment turns the cache off (every release is a cudaFree).
bool cache_enabled() {
    static const bool on = [] {
        const char* v = std::getenv("SB_DEVICE_CACHE");
        return !(v && v[0] == '0');
    }();
    return on;
}

size_t round_block(size_t n) {
    const size_t g = n >= (size_t(1) << 20) ? (size_t(2) << 20) : 512;
    return (n + g - 1) / g * g;
}

void trim_locked(int device) {
    int cur = 0;
    cudaGetDevice(&cur);
    for (auto it = g_free.begin(); it != g_free.end();) {
        if (device >= 0 && it->first.first != device) {
            ++it;
            continue;
        }
        cudaSetDevice(it->first.first);
        for (void* q : it->second) cudaFree(q);
        g_cached[it->first.first] -= static_cast<int64_t>(it->first.second * it->second.size());
        it = g_free.erase(it);
    }
    cudaSetDevice(cur);
}
}  // namespace

void h2d_sync(void* dst, const void* src, size_t bytes) {
    SB_CUDA(cudaMemcpy(dst, src, bytes, cudaMemcpyHostToDevice));
    SB_CUDA(cudaStreamSynchronize(0));
}

void memset_sync(void* dst, int value, size_t bytes) {
    SB_CUDA(cudaMemset(dst, value, bytes));
    SB_CUDA(cudaStreamSynchronize(0));
}

void memory_trim(int device) {
    std::lock_guard<std::mutex> lock(g_mem_mu);
    trim_locked(device);
}

void memory_stats(int device, int64_t* in_use, int64_t* cached) {
    std::lock_guard<std::mutex> lock(g_mem_mu);
    if (in_use) *in_use = g_in_use[device];
    if (cached) *cached = g_cached[device];
}

void DevBuf::alloc(size_t n) {
    release();
    if (n == 0) n = 16;
    maybe_inject(SB_INJECT_ALLOC);
    int device = 0;
    SB_CUDA(cudaGetDevice(&device));
    const size_t c = round_block(n);
    std::lock_guard<std::mutex> lock(g_mem_mu);
    auto it = g_free.find({device, c});
    if (it != g_free.end() && !it->second.empty()) {
        p = it->second.back();
        it->second.pop_back();
        g_cached[device] -= static_cast<int64_t>(c);
    } else {
        cudaError_t e = cudaMalloc(&p, c);
        if (e == cudaErrorMemoryAllocation) {
            cudaGetLastError();
            trim_locked(-1);
            e = cudaMalloc(&p, c);
        }
        if (e != cudaSuccess) {
            p = nullptr;
            cudaGetLastError();
            throw Error{e == cudaErrorMemoryAllocation ? SB_ERR_OUT_OF_MEMORY : SB_ERR_CUDA,
                        std::string("device allocation of ") + std::to_string(n) + " bytes failed: " +
                            cudaGetErrorString(e)};
        }
    }
    bytes = n;
    cap = c;
    dev = device;
    g_in_use[device] += static_cast<int64_t>(c);
}

void DevBuf::release() {
    if (!p) return;
    std::lock_guard<std::mutex> lock(g_mem_mu);
    int cur = 0;
    cudaGetDevice(&cur);
    if (cur != dev) cudaSetDevice(dev);
    g_in_use[dev] -= static_cast<int64_t>(cap);
    // Work still queued on any stream may use the block: wait for the device, as cudaFree does.
    if (cache_enabled() && cudaDeviceSynchronize() == cudaSuccess &&
        g_cached[dev] + static_cast<int64_t>(cap) <= static_cast<int64_t>(kCacheLimit)) {
        g_free[{dev, cap}].push_back(p);
        g_cached[dev] += static_cast<int64_t>(cap);
    } else {
        cudaGetLastError();
        cudaFree(p);
    }
    if (cur != dev) cudaSetDevice(cur);
    p = nullptr;
    bytes = cap = 0;
    dev = -1;
}

int device_sm_count(int device) {
    int v = 0;
    cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, device);
    return v;
}

template <class F>
static int guarded(F&& f) {
    return abi_guard(std::forward<F>(f));
}

static bool all_finite(const sb_complex* v, int64_t n) {
    for (int64_t i = 0; i < n; ++i)
        if (!std::isfinite(v[i].re) || !std::isfinite(v[i].im)) return false;
    return true;
}

static int64_t icosphere_tris(int level) {
    int64_t f = 20;
    for (int i = 0; i < level; ++i) f *= 4;
    return f;
}

}  // namespace sb

using namespace sb;

extern "C" {

SB_API int sb_last_error(char* buf, size_t len) {
    if (buf && len) {
        std::strncpy(buf, t_err.c_str(), len - 1);
        buf[len - 1] = '\0';
    }
    return static_cast<int>(t_err.size());
}

SB_API int sb_version(int* major, int* minor, int* patch) {
    if (major) *major = 0;
    if (minor) *minor = 1;
    if (patch) *patch = 0;
    return SB_OK;
}

SB_API int sb_device_count(int* count) {
    return guarded([&] {
        SB_REQUIRE(count, SB_ERR_INVALID_ARGUMENT, "null count");
        int n = 0;
        cudaError_t e = cudaGetDeviceCount(&n);
        if (e != cudaSuccess) {
            cudaGetLastError();
            n = 0;
        }
        *count = n;
    });
}

SB_API int sb_physics_new(double frequency, double c, double rho, int is_internal, sb_physics* out) {
    return guarded([&] {
        SB_REQUIRE(out, SB_ERR_INVALID_ARGUMENT, "null output");
        SB_REQUIRE(std::isfinite(frequency) && frequency > 0, SB_ERR_INVALID_ARGUMENT, "frequency must be finite and positive");
        SB_REQUIRE(std::isfinite(c) && c > 0, SB_ERR_INVALID_ARGUMENT, "speed_of_sound must be finite and positive");
        SB_REQUIRE(std::isfinite(rho) && rho > 0, SB_ERR_INVALID_ARGUMENT, "density must be finite and positive");
        const double omega = 2.0 * 3.14159265358979323846 * frequency;
        out->frequency = frequency;
        out->speed_of_sound = c;
        out->density = rho;
        out->omega = omega;
        out->wave_number = omega / c;
        out->wave_length = c / frequency;
        out->harmonic_factor = 1.0;
        out->pressure_factor = rho * omega * 1.0;
        out->tau = is_internal ? -1.0 : 1.0;
    });
}

SB_API int sb_physics_validate(const sb_physics* p) {
    return guarded([&] {
        SB_REQUIRE(p, SB_ERR_INVALID_ARGUMENT, "null physics");
        SB_REQUIRE(std::isfinite(p->frequency) && p->frequency > 0, SB_ERR_INVALID_ARGUMENT, "invalid frequency");
        SB_REQUIRE(std::isfinite(p->speed_of_sound) && p->speed_of_sound > 0, SB_ERR_INVALID_ARGUMENT, "invalid speed_of_sound");
        SB_REQUIRE(std::isfinite(p->density) && p->density > 0, SB_ERR_INVALID_ARGUMENT, "invalid density");
        SB_REQUIRE(p->harmonic_factor == 1.0 || p->harmonic_factor == -1.0, SB_ERR_INVALID_ARGUMENT, "invalid harmonic_factor");
        SB_REQUIRE(p->tau == 1.0 || p->tau == -1.0, SB_ERR_INVALID_ARGUMENT, "invalid tau");
        const double omega = 2.0 * 3.14159265358979323846 * p->frequency;
        auto close = [](double a, double b) {
            return std::isfinite(a) && std::fabs(a - b) <= 1e-12 * std::fmax(std::fmax(std::fabs(a), std::fabs(b)), 1.0);
        };
        SB_REQUIRE(close(p->omega, omega), SB_ERR_INVALID_ARGUMENT, "inconsistent omega");
        SB_REQUIRE(close(p->wave_number, omega / p->speed_of_sound), SB_ERR_INVALID_ARGUMENT, "inconsistent wave_number");
        SB_REQUIRE(close(p->pressure_factor, p->density * omega * p->harmonic_factor), SB_ERR_INVALID_ARGUMENT,
                   "inconsistent pressure_factor");
    });
}

SB_API int sb_burton_miller_beta(const sb_physics* p, double scale, sb_complex* beta) {
    return guarded([&] {
        SB_REQUIRE(p && beta, SB_ERR_INVALID_ARGUMENT, "null argument");
        beta->re = 0.0;
        beta->im = p->tau > 0.0 ? scale * p->harmonic_factor / p->wave_number : 0.0;
    });
}

SB_API int sb_icosphere_counts(int level, int64_t* n_nodes, int64_t* n_tris) {
    return guarded([&] {
        SB_REQUIRE(level >= 0 && level <= 9, SB_ERR_INVALID_ARGUMENT, "icosphere level must be 0..9");
        SB_REQUIRE(n_nodes && n_tris, SB_ERR_INVALID_ARGUMENT, "null output");
        *n_tris = icosphere_tris(level);
        *n_nodes = *n_tris / 2 + 2;
    });
}

// generate_icosphere_mesh (crates/sonium-bem/src/core/mesh/generators.rs:309-397): the
// golden-ratio icosahedron (12 vertices, 20 faces in the reference's order) subdivided `level`
// times with edge midpoints projected to the unit sphere, children (v0, m01, m20), (v1, m12, m01),
// (v2, m20, m12), (m01, m12, m20), then scaled by the radius (and per axis by `scale`).
SB_API int sb_icosphere(double radius, int level, const double* scale, double* nodes, uint32_t* tris) {
    return guarded([&] {
        SB_REQUIRE(level >= 0 && level <= 9, SB_ERR_INVALID_ARGUMENT, "icosphere level must be 0..9");
        SB_REQUIRE(nodes && tris, SB_ERR_INVALID_ARGUMENT, "null output");
        SB_REQUIRE(std::isfinite(radius) && radius > 0, SB_ERR_INVALID_ARGUMENT, "radius must be positive");
        const double phi = (1.0 + std::sqrt(5.0)) / 2.0;
        std::vector<double> v = {-1, phi, 0, 1, phi, 0, -1, -phi, 0, 1, -phi, 0, 0, -1, phi, 0, 1, phi,
                                 0, -1, -phi, 0, 1, -phi, phi, 0, -1, phi, 0, 1, -phi, 0, -1, -phi, 0, 1};
        for (size_t i = 0; i < 12; ++i) {
            double* p = &v[3 * i];
            const double len = std::sqrt(p[0] * p[0] + p[1] * p[1] + p[2] * p[2]);
            p[0] /= len;
            p[1] /= len;
            p[2] /= len;
        }
        std::vector<uint32_t> f = {0, 11, 5, 0, 5, 1, 0, 1, 7, 0, 7, 10, 0, 10, 11, 1, 5, 9, 5, 11, 4,
                                   11, 10, 2, 10, 7, 6, 7, 1, 8, 3, 9, 4, 3, 4, 2, 3, 2, 6, 3, 6, 8,
                                   3, 8, 9, 4, 9, 5, 2, 4, 11, 6, 2, 10, 8, 6, 7, 9, 8, 1};
        for (int l = 0; l < level; ++l) {
            const size_t nv0 = v.size() / 3;
            std::vector<std::vector<std::pair<uint32_t, uint32_t>>> cache(nv0);
            auto mid = [&](uint32_t a, uint32_t b) -> uint32_t {
                const uint32_t lo = std::min(a, b), hi = std::max(a, b);
                for (auto& kv : cache[lo])
                    if (kv.first == hi) return kv.second;
                double m[3] = {(v[3 * a] + v[3 * b]) / 2.0, (v[3 * a + 1] + v[3 * b + 1]) / 2.0,
                               (v[3 * a + 2] + v[3 * b + 2]) / 2.0};
                const double len = std::sqrt(m[0] * m[0] + m[1] * m[1] + m[2] * m[2]);
                const uint32_t idx = static_cast<uint32_t>(v.size() / 3);
                v.push_back(m[0] / len);
                v.push_back(m[1] / len);
                v.push_back(m[2] / len);
                cache[lo].push_back({hi, idx});
                return idx;
            };
            std::vector<uint32_t> nf;
            nf.reserve(f.size() * 4);
            for (size_t t = 0; t < f.size() / 3; ++t) {
                const uint32_t a = f[3 * t], b = f[3 * t + 1], c = f[3 * t + 2];
                const uint32_t m01 = mid(a, b), m12 = mid(b, c), m20 = mid(c, a);
                const uint32_t add[12] = {a, m01, m20, b, m12, m01, c, m20, m12, m01, m12, m20};
                nf.insert(nf.end(), add, add + 12);
            }
            f.swap(nf);
        }
        const double sx = scale ? scale[0] : 1.0, sy = scale ? scale[1] : 1.0, sz = scale ? scale[2] : 1.0;
        for (size_t i = 0; i < v.size() / 3; ++i) {
            nodes[3 * i] = v[3 * i] * radius * sx;
            nodes[3 * i + 1] = v[3 * i + 1] * radius * sy;
            nodes[3 * i + 2] = v[3 * i + 2] * radius * sz;
        }
        std::memcpy(tris, f.data(), sizeof(uint32_t) * f.size());
    });
}

SB_API int sb_mesh_create(const double* nodes, int64_t n_nodes, const uint32_t* tris, int64_t n_tris,
                          int device, sb_mesh** out) {
    return guarded([&] {
        SB_REQUIRE(out, SB_ERR_INVALID_ARGUMENT, "null output handle");
        *out = nullptr;
        Mesh* m = mesh_create(nodes, n_nodes, tris, n_tris, device);
        *out = new sb_mesh{m};
    });
}

SB_API int sb_mesh_create_quad4(const double* nodes, int64_t n_nodes, const uint32_t* quads, int64_t n_quads,
                                int device, sb_mesh** out) {
    return guarded([&] {
        SB_REQUIRE(out, SB_ERR_INVALID_ARGUMENT, "null output handle");
        *out = nullptr;
        Mesh* m = mesh_create_quad(nodes, n_nodes, quads, n_quads, device);
        *out = new sb_mesh{m};
    });
}

SB_API int sb_mesh_destroy(sb_mesh* mesh) {
    return guarded([&] {
        if (!mesh) return;
        if (mesh->m) {
            cudaSetDevice(mesh->m->device);
            delete mesh->m;
        }
        delete mesh;
    });
}

SB_API int sb_mesh_info_get(const sb_mesh* mesh, sb_mesh_info* info) {
    return guarded([&] {
        SB_REQUIRE(mesh && mesh->m && info, SB_ERR_INVALID_ARGUMENT, "null argument");
        info->n_nodes = mesh->m->n_nodes;
        info->n_elements = mesh->m->n;
        info->n_near_pairs = mesh->m->nnz;
        info->device = mesh->m->device;
        info->reserved = 0;
    });
}

SB_API int sb_mesh_element_geometry(const sb_mesh* mesh, double* centers, double* normals, double* areas) {
    return guarded([&] {
        SB_REQUIRE(mesh && mesh->m, SB_ERR_INVALID_ARGUMENT, "null mesh");
        const Mesh& m = *mesh->m;
        const std::vector<double>& he = mesh_host_elem(m);
        for (int64_t e = 0; e < m.n; ++e) {
            for (int c = 0; c < 3; ++c) {
                if (centers) centers[3 * e + c] = he[(ECX + c) * m.ld + e];
                if (normals) normals[3 * e + c] = he[(ENX + c) * m.ld + e];
            }
            if (areas) areas[e] = he[EAREA * m.ld + e];
        }
    });
}

SB_API int sb_mesh_set_bc(sb_mesh* mesh, const int32_t* kind, const sb_complex* value,
                          const uint8_t* has_admittance, const sb_complex* admittance) {
    return guarded([&] {
        SB_REQUIRE(mesh && mesh->m, SB_ERR_INVALID_ARGUMENT, "null mesh");
        mesh_set_bc(*mesh->m, kind, value, has_admittance, admittance);
    });
}

static void check_beta(sb_complex beta) {
    SB_REQUIRE(std::isfinite(beta.re) && std::isfinite(beta.im), SB_ERR_INVALID_ARGUMENT, "beta must be finite");
}

SB_API int sb_assemble(const sb_mesh* mesh, const sb_physics* physics, sb_complex beta, int precision,
                       sb_operator** out) {
    return guarded([&] {
        SB_REQUIRE(mesh && mesh->m && physics && out, SB_ERR_INVALID_ARGUMENT, "null argument");
        *out = nullptr;
        SB_REQUIRE(precision == SB_PRECISION_FP64 || precision == SB_PRECISION_FP64_FP32 ||
                       precision == SB_PRECISION_FP32 || precision == SB_PRECISION_FP32_HALF,
                   SB_ERR_INVALID_ARGUMENT, "unknown precision");
        SB_REQUIRE(sb_physics_validate(physics) == SB_OK, SB_ERR_INVALID_ARGUMENT, "invalid physics: " + t_err);
        check_beta(beta);
        const bool half = precision == SB_PRECISION_FP32_HALF;
        if (half) precision = SB_PRECISION_FP32;
        Mesh& m = *mesh->m;
        SB_REQUIRE(!m.quad || precision == SB_PRECISION_FP64, SB_ERR_INVALID_ARGUMENT,
                   "Quad4 mesh: only SB_PRECISION_FP64 is supported");
        if (!m.bc_kind.p) mesh_set_bc(m, nullptr, nullptr, nullptr, nullptr);
        SB_CUDA(cudaSetDevice(m.device));
        Operator* op = new Operator();
        try {
            op->mesh = &m;
            op->device = m.device;
            op->precision = precision;
            op->n = m.n;
            op->lda32 = (m.n + 1) / 2 * 2;
            SB_CUDA(cudaStreamCreateWithFlags(&op->stream, cudaStreamNonBlocking));
            if (precision != SB_PRECISION_FP32) op->A64.alloc(sizeof(double2) * m.n * m.n);
            if (precision != SB_PRECISION_FP64) op->A32.alloc(sizeof(float2) * m.n * op->lda32);
            if (half) op->inner = SB_INNER_FP16;
            assemble(*op, *physics, beta.re, beta.im);
        } catch (...) {
            if (op->stream) cudaStreamDestroy(op->stream);
            delete op;
            throw;
        }
        *out = new sb_operator{op};
    });
}

SB_API int sb_operator_from_dense(int device, int64_t n, const sb_complex* matrix, int precision, sb_operator** out) {
    return guarded([&] {
        SB_REQUIRE(matrix && out, SB_ERR_INVALID_ARGUMENT, "null argument");
        *out = nullptr;
        SB_REQUIRE(n > 0, SB_ERR_INVALID_ARGUMENT, "dense operator: n must be positive");
        SB_REQUIRE(precision == SB_PRECISION_FP64 || precision == SB_PRECISION_FP64_FP32 ||
                       precision == SB_PRECISION_FP32,
                   SB_ERR_INVALID_ARGUMENT, "unknown precision");
        int count = 0;
        SB_CUDA(cudaGetDeviceCount(&count));
        SB_REQUIRE(device >= 0 && device < count, SB_ERR_INVALID_ARGUMENT, "no such device");
        SB_REQUIRE(all_finite(matrix, n * n), SB_ERR_NOT_FINITE, "dense operator: non-finite matrix entry");
        SB_CUDA(cudaSetDevice(device));
        Operator* op = new Operator();
        try {
            op->device = device;
            op->precision = precision;
            op->n = n;
            op->lda32 = (n + 1) / 2 * 2;
            SB_CUDA(cudaStreamCreateWithFlags(&op->stream, cudaStreamNonBlocking));
            if (precision != SB_PRECISION_FP32) {
                op->A64.alloc(sizeof(double2) * n * n);
                h2d_sync(op->A64.p, matrix, sizeof(double2) * n * n);
            }
            if (precision != SB_PRECISION_FP64) {
                op->A32.alloc(sizeof(float2) * n * op->lda32);
                std::vector<float2> row(op->lda32, make_float2(0.f, 0.f));
                for (int64_t i = 0; i < n; ++i) {
                    for (int64_t j = 0; j < n; ++j)
                        row[j] = make_float2(static_cast<float>(matrix[i * n + j].re),
                                             static_cast<float>(matrix[i * n + j].im));
                    SB_CUDA(cudaMemcpy(op->A32.as<float2>() + i * op->lda32, row.data(), sizeof(float2) * op->lda32,
                                       cudaMemcpyHostToDevice)); SB_CUDA(cudaStreamSynchronize(0));
                }
            }
            std::vector<sb_complex> d(n);
            for (int64_t i = 0; i < n; ++i) d[i] = matrix[i * n + i];
            op->diag.alloc(sizeof(double2) * n);
            h2d_sync(op->diag.p, d.data(), sizeof(double2) * n);
            op->rhs.alloc(sizeof(double2) * n);
            memset_sync(op->rhs.p, 0, sizeof(double2) * n);
        } catch (...) {
            if (op->stream) cudaStreamDestroy(op->stream);
            delete op;
            throw;
        }
        *out = new sb_operator{op};
    });
}

SB_API int sb_assemble_into(sb_operator* op, const sb_physics* physics, sb_complex beta) {
    return guarded([&] {
        SB_REQUIRE(op && op->op && physics, SB_ERR_INVALID_ARGUMENT, "null argument");
        SB_REQUIRE(op->op->mesh, SB_ERR_INVALID_ARGUMENT, "operator was not assembled from a mesh");
        SB_REQUIRE(sb_physics_validate(physics) == SB_OK, SB_ERR_INVALID_ARGUMENT, "invalid physics: " + t_err);
        check_beta(beta);
        tensor_release(*op->op);
        op->op->half_valid = false;
        op->op->bj_valid = false;
        op->op->bj64_valid = false;
        if (op->op->basis != SB_BASIS_CONSTANT)
            assemble_discontinuous(*op->op, *physics, beta.re, beta.im);
        else
            assemble(*op->op, *physics, beta.re, beta.im);
    });
}

static void create_discontinuous(const sb_mesh* mesh, const sb_physics* physics, sb_complex beta, int basis,
                                 double sign, sb_operator** out) {
        SB_REQUIRE(mesh && mesh->m && physics && out, SB_ERR_INVALID_ARGUMENT, "null argument");
        *out = nullptr;
        SB_REQUIRE(!mesh->m->quad, SB_ERR_UNSUPPORTED_ELEMENT, "discontinuous bases: Tri3 meshes only");
        SB_REQUIRE(basis == SB_BASIS_LINEAR || basis == SB_BASIS_QUADRATIC, SB_ERR_INVALID_ARGUMENT,
                   "discontinuous basis must be SB_BASIS_LINEAR or SB_BASIS_QUADRATIC");
        SB_REQUIRE(sign == 1.0 || sign == -1.0, SB_ERR_INVALID_ARGUMENT, "sign must be +1 or -1");
        SB_REQUIRE(sb_physics_validate(physics) == SB_OK, SB_ERR_INVALID_ARGUMENT, "invalid physics: " + t_err);
        check_beta(beta);
        Mesh& m = *mesh->m;
        if (!m.bc_kind.p) mesh_set_bc(m, nullptr, nullptr, nullptr, nullptr);
        SB_REQUIRE(!m.any_bc_value, SB_ERR_INVALID_ARGUMENT,
                   "linear basis: prescribed boundary values are not supported (rigid, zero-pressure or "
                   "admittance surfaces)");
        SB_CUDA(cudaSetDevice(m.device));
        Operator* op = new Operator();
        try {
            op->mesh = &m;
            op->device = m.device;
            op->precision = SB_PRECISION_FP64;
            op->basis = basis;
            op->sign = sign;
            op->n = (basis == SB_BASIS_QUADRATIC ? 6 : 3) * m.n;
            op->lda32 = (op->n + 1) / 2 * 2;
            SB_CUDA(cudaStreamCreateWithFlags(&op->stream, cudaStreamNonBlocking));
            op->A64.alloc(sizeof(double2) * op->n * op->n);
            assemble_discontinuous(*op, *physics, beta.re, beta.im);
        } catch (...) {
            if (op->stream) cudaStreamDestroy(op->stream);
            delete op;
            throw;
        }
        *out = new sb_operator{op};
}

SB_API int sb_assemble_linear(const sb_mesh* mesh, const sb_physics* physics, sb_complex beta, sb_operator** out) {
    return guarded([&] { create_discontinuous(mesh, physics, beta, SB_BASIS_LINEAR, 1.0, out); });
}

SB_API int sb_assemble_discontinuous(const sb_mesh* mesh, const sb_physics* physics, sb_complex beta, int basis,
                                     double sign, sb_operator** out) {
    return guarded([&] { create_discontinuous(mesh, physics, beta, basis, sign, out); });
}

SB_API int sb_mesh_collocation(const sb_mesh* mesh, int basis, double* points, double* normals) {
    return guarded([&] {
        SB_REQUIRE(mesh && mesh->m && points && normals, SB_ERR_INVALID_ARGUMENT, "null argument");
        SB_REQUIRE(basis == SB_BASIS_CONSTANT || basis == SB_BASIS_LINEAR || basis == SB_BASIS_QUADRATIC,
                   SB_ERR_INVALID_ARGUMENT, "unknown basis");
        const Mesh& m = *mesh->m;
        SB_REQUIRE(basis == SB_BASIS_CONSTANT || !m.quad, SB_ERR_UNSUPPORTED_ELEMENT,
                   "discontinuous bases: Tri3 meshes only");
        if (basis == SB_BASIS_CONSTANT) {
            const std::vector<double>& he = mesh_host_elem(m);
            for (int64_t e = 0; e < m.n; ++e)
                for (int c = 0; c < 3; ++c) {
                    points[3 * e + c] = he[(ECX + c) * m.ld + e];
                    normals[3 * e + c] = he[(ENX + c) * m.ld + e];
                }
            return;
        }
        // The discontinuous rows' points from the assembly's kernel.
        SB_CUDA(cudaSetDevice(m.device));
        const int64_t n3 = (basis == SB_BASIS_QUADRATIC ? 6 : 3) * m.n;
        DevBuf dcp, dcn;
        dcp.alloc(sizeof(double) * 3 * n3);
        dcn.alloc(sizeof(double) * 3 * n3);
        lin_collocation(m, basis, dcp.as<double>(), dcn.as<double>());
        std::vector<double> cp(3 * n3), cn(3 * n3);
        SB_CUDA(cudaMemcpy(cp.data(), dcp.p, sizeof(double) * 3 * n3, cudaMemcpyDeviceToHost));
        SB_CUDA(cudaMemcpy(cn.data(), dcn.p, sizeof(double) * 3 * n3, cudaMemcpyDeviceToHost));
        for (int64_t r = 0; r < n3; ++r)
            for (int c = 0; c < 3; ++c) {
                points[3 * r + c] = cp[c * n3 + r];
                normals[3 * r + c] = cn[c * n3 + r];
            }
    });
}

SB_API int sb_rhs_plane_wave_points(int device, int64_t np, const double* points, const double* normals,
                                    const sb_physics* physics, sb_complex beta, const double* dirs,
                                    const sb_complex* amps, int64_t r, sb_complex* rhs) {
    return guarded([&] {
        SB_REQUIRE(points && normals && physics && dirs && rhs && np >= 1 && r >= 1, SB_ERR_INVALID_ARGUMENT,
                   "bad argument");
        SB_REQUIRE(sb_physics_validate(physics) == SB_OK, SB_ERR_INVALID_ARGUMENT, "invalid physics: " + t_err);
        check_beta(beta);
        for (int64_t q = 0; q < 3 * r; ++q)
            SB_REQUIRE(std::isfinite(dirs[q]), SB_ERR_INVALID_ARGUMENT, "non-finite direction");
        for (int64_t i = 0; i < 3 * np; ++i)
            SB_REQUIRE(std::isfinite(points[i]) && std::isfinite(normals[i]), SB_ERR_NOT_FINITE,
                       "non-finite collocation point or normal");
        int count = 0;
        SB_CUDA(cudaGetDeviceCount(&count));
        SB_REQUIRE(device >= 0 && device < count, SB_ERR_INVALID_ARGUMENT, "no such device");
        SB_CUDA(cudaSetDevice(device));
        std::vector<double> soa(6 * np);
        for (int64_t i = 0; i < np; ++i)
            for (int c = 0; c < 3; ++c) {
                soa[c * np + i] = points[3 * i + c];
                soa[(3 + c) * np + i] = normals[3 * i + c];
            }
        DevBuf dp, dr;
        dp.alloc(sizeof(double) * 6 * np);
        dr.alloc(sizeof(double2) * np * r);
        h2d_sync(dp.p, soa.data(), sizeof(double) * 6 * np);
        incident_plane_wave_at(device, dp.as<double>(), dp.as<double>() + 3 * np, np, np, *physics, beta.re, beta.im,
                               dirs, reinterpret_cast<const double*>(amps), r, dr.as<double2>(), 0);
        SB_CUDA(cudaMemcpy(rhs, dr.p, sizeof(double2) * np * r, cudaMemcpyDeviceToHost));
    });
}

SB_API int sb_operator_destroy(sb_operator* op) {
    return guarded([&] {
        if (!op) return;
        if (op->op) {
            cudaSetDevice(op->op->device);
            destroy_solve_work(*op->op);
            multi_release(*op->op);
            tensor_release(*op->op);
            op->op->side.release();
            if (op->op->stream) cudaStreamDestroy(op->op->stream);
            delete op->op;
        }
        delete op;
    });
}

SB_API int sb_operator_info_get(const sb_operator* op, sb_operator_info* info) {
    return guarded([&] {
        SB_REQUIRE(op && op->op && info, SB_ERR_INVALID_ARGUMENT, "null argument");
        info->n = op->op->n;
        info->precision = op->op->precision;
        info->device = op->op->device;
        info->assembly_ms = op->op->last_assembly_ms;
        info->bytes_fp64 = op->op->A64.bytes;
        info->bytes_fp32 = op->op->A32.bytes;
    });
}

SB_API int sb_operator_copy_to_host(const sb_operator* op, sb_complex* matrix, sb_complex* rhs) {
    return guarded([&] {
        SB_REQUIRE(op && op->op, SB_ERR_INVALID_ARGUMENT, "null operator");
        const Operator& o = *op->op;
        SB_CUDA(cudaSetDevice(o.device));
        SB_CUDA(cudaStreamSynchronize(o.stream));
        if (matrix && o.A64.p) {
            SB_CUDA(cudaMemcpy(matrix, o.A64.p, sizeof(double2) * o.n * o.n, cudaMemcpyDeviceToHost));
        } else if (matrix) {
            // complex64-only operator: widen its entries
            std::vector<float2> row(o.n);
            for (int64_t i = 0; i < o.n; ++i) {
                SB_CUDA(cudaMemcpy(row.data(), o.A32.as<float2>() + i * o.lda32, sizeof(float2) * o.n,
                                   cudaMemcpyDeviceToHost));
                for (int64_t j = 0; j < o.n; ++j) matrix[i * o.n + j] = sb_complex{row[j].x, row[j].y};
            }
        }
        if (rhs) SB_CUDA(cudaMemcpy(rhs, o.rhs.p, sizeof(double2) * o.n, cudaMemcpyDeviceToHost));
    });
}

SB_API int sb_operator_copy_rows_to_host(const sb_operator* op, int64_t row0, int64_t row1, sb_complex* rows) {
    return guarded([&] {
        SB_REQUIRE(op && op->op && rows, SB_ERR_INVALID_ARGUMENT, "null argument");
        const Operator& o = *op->op;
        SB_REQUIRE(row0 >= 0 && row1 <= o.n && row0 <= row1, SB_ERR_INVALID_ARGUMENT, "row range out of bounds");
        SB_CUDA(cudaSetDevice(o.device));
        SB_CUDA(cudaStreamSynchronize(o.stream));
        if (o.A64.p) {
            SB_CUDA(cudaMemcpy(rows, o.A64.as<double2>() + row0 * o.n, sizeof(double2) * (row1 - row0) * o.n,
                               cudaMemcpyDeviceToHost));
        } else {
            std::vector<float2> row(o.n);
            for (int64_t i = row0; i < row1; ++i) {
                SB_CUDA(cudaMemcpy(row.data(), o.A32.as<float2>() + i * o.lda32, sizeof(float2) * o.n,
                                   cudaMemcpyDeviceToHost));
                for (int64_t j = 0; j < o.n; ++j) rows[(i - row0) * o.n + j] = sb_complex{row[j].x, row[j].y};
            }
        }
    });
}

SB_API int sb_operator_copy_to_host_c64(const sb_operator* op, sb_complex32* matrix) {
    return guarded([&] {
        SB_REQUIRE(op && op->op && matrix, SB_ERR_INVALID_ARGUMENT, "null argument");
        const Operator& o = *op->op;
        SB_REQUIRE(o.A32.p, SB_ERR_INVALID_ARGUMENT, "operator has no complex64 copy");
        SB_CUDA(cudaSetDevice(o.device));
        SB_CUDA(cudaStreamSynchronize(o.stream));
        SB_CUDA(cudaMemcpy2D(matrix, sizeof(float2) * o.n, o.A32.p, sizeof(float2) * o.lda32, sizeof(float2) * o.n,
                             o.n, cudaMemcpyDeviceToHost));
    });
}

// op(A) x with FP64 vectors; transposed products need the complex128 matrix.
static void apply_any(Operator& o, Trans t, const double2* x, double2* y) {
    if (t == Trans::N) {
        op_gemv64(o, x, y, Gate{});
        return;
    }
    SB_REQUIRE(o.A64.p, SB_ERR_INVALID_ARGUMENT,
               "transposed products need the complex128 matrix (SB_PRECISION_FP64 or SB_PRECISION_FP64_FP32)");
    gemv_c128(o.A64.as<double2>(), o.n, x, y, t, o.stream, o.scratch);
}

static Trans to_trans(int t) {
    SB_REQUIRE(t == SB_OP_N || t == SB_OP_T || t == SB_OP_C, SB_ERR_INVALID_ARGUMENT, "trans must be N, T or C");
    return static_cast<Trans>(t);
}

SB_API int sb_operator_apply_device(const sb_operator* op, int trans, const sb_complex* x_dev, sb_complex* y_dev) {
    return guarded([&] {
        SB_REQUIRE(op && op->op && x_dev && y_dev, SB_ERR_INVALID_ARGUMENT, "null argument");
        Operator& o = *op->op;
        SB_CUDA(cudaSetDevice(o.device));
        maybe_inject(SB_INJECT_LAUNCH);
        apply_any(o, to_trans(trans), reinterpret_cast<const double2*>(x_dev), reinterpret_cast<double2*>(y_dev));
        SB_CUDA(cudaStreamSynchronize(o.stream));
    });
}

SB_API int sb_operator_apply(const sb_operator* op, int trans, const sb_complex* x, sb_complex* y) {
    return guarded([&] {
        SB_REQUIRE(op && op->op && x && y, SB_ERR_INVALID_ARGUMENT, "null argument");
        Operator& o = *op->op;
        const Trans t = to_trans(trans);
        SB_REQUIRE(all_finite(x, o.n), SB_ERR_NOT_FINITE, "apply: non-finite input vector");
        SB_CUDA(cudaSetDevice(o.device));
        maybe_inject(SB_INJECT_LAUNCH);
        DevBuf dx, dy;
        dx.alloc(sizeof(double2) * o.n);
        dy.alloc(sizeof(double2) * o.n);
        SB_CUDA(cudaMemcpyAsync(dx.p, x, sizeof(double2) * o.n, cudaMemcpyHostToDevice, o.stream));
        apply_any(o, t, dx.as<double2>(), dy.as<double2>());
        SB_CUDA(cudaMemcpyAsync(y, dy.p, sizeof(double2) * o.n, cudaMemcpyDeviceToHost, o.stream));
        SB_CUDA(cudaStreamSynchronize(o.stream));
        SB_REQUIRE(all_finite(y, o.n), SB_ERR_NOT_FINITE, "apply: non-finite output vector");
    });
}

SB_API int sb_operator_apply_block(const sb_operator* op, const sb_complex* X, sb_complex* Y, int64_t r) {
    return guarded([&] {
        SB_REQUIRE(op && op->op && X && Y && r >= 1, SB_ERR_INVALID_ARGUMENT, "bad argument");
        Operator& o = *op->op;
        const int64_t n = o.n;
        SB_REQUIRE(all_finite(X, n * r), SB_ERR_NOT_FINITE, "apply_block: non-finite input block");
        SB_CUDA(cudaSetDevice(o.device));
        maybe_inject(SB_INJECT_LAUNCH);
        // Column-at-a-time products over the row-major block (gathered on the host).
        DevBuf dx, dy;
        dx.alloc(sizeof(double2) * n);
        dy.alloc(sizeof(double2) * n);
        std::vector<sb_complex> col(n);
        for (int64_t q = 0; q < r; ++q) {
            for (int64_t i = 0; i < n; ++i) col[i] = X[i * r + q];
            SB_CUDA(cudaMemcpyAsync(dx.p, col.data(), sizeof(double2) * n, cudaMemcpyHostToDevice, o.stream));
            apply_any(o, Trans::N, dx.as<double2>(), dy.as<double2>());
            SB_CUDA(cudaMemcpyAsync(col.data(), dy.p, sizeof(double2) * n, cudaMemcpyDeviceToHost, o.stream));
            SB_CUDA(cudaStreamSynchronize(o.stream));
            for (int64_t i = 0; i < n; ++i) Y[i * r + q] = col[i];
        }
        SB_REQUIRE(all_finite(Y, n * r), SB_ERR_NOT_FINITE, "apply_block: non-finite output block");
    });
}

SB_API int sb_operator_prepare_block_tensor(sb_operator* op) {
    return guarded([&] {
        SB_REQUIRE(op && op->op, SB_ERR_INVALID_ARGUMENT, "null operator");
        maybe_inject(SB_INJECT_LAUNCH);
        tensor_prepare(*op->op);
    });
}

SB_API int sb_operator_apply_block_tensor(const sb_operator* op, const sb_complex32* x, sb_complex32* y, int64_t r) {
    return guarded([&] {
        SB_REQUIRE(op && op->op && x && y && r >= 1, SB_ERR_INVALID_ARGUMENT, "bad argument");
        SB_REQUIRE(r <= (int64_t)1 << 20, SB_ERR_INVALID_ARGUMENT, "apply_block_tensor: too many vectors");
        Operator& o = *op->op;
        const int64_t n = o.n;
        for (int64_t t = 0; t < n * r; ++t)
            SB_REQUIRE(std::isfinite(x[t].re) && std::isfinite(x[t].im), SB_ERR_NOT_FINITE,
                       "apply_block_tensor: non-finite input block");
        SB_CUDA(cudaSetDevice(o.device));
        maybe_inject(SB_INJECT_LAUNCH);
        DevBuf dx, dy;
        dx.alloc(sizeof(float2) * n * r);
        dy.alloc(sizeof(float2) * n * r);
        SB_CUDA(cudaMemcpyAsync(dx.p, x, sizeof(float2) * n * r, cudaMemcpyHostToDevice, o.stream));
        tensor_block_product(o, dx.as<float2>(), n, static_cast<int>(r), dy.as<float2>(), n, o.stream);
        SB_CUDA(cudaMemcpyAsync(y, dy.p, sizeof(float2) * n * r, cudaMemcpyDeviceToHost, o.stream));
        SB_CUDA(cudaStreamSynchronize(o.stream));
        SB_REQUIRE(tensor_status(o, true) == 0, SB_ERR_DEVICE_CHECK,
                   "apply_block_tensor: a pipeline wait of the tensor-core kernel timed out");
    });
}

static void check_ir(const sb_ir_config* cfg);

SB_API int sb_operator_apply_block_tensor_device(const sb_operator* op, const sb_complex32* x_dev,
                                                 sb_complex32* y_dev, int64_t r) {
    return guarded([&] {
        SB_REQUIRE(op && op->op && x_dev && y_dev && r >= 1, SB_ERR_INVALID_ARGUMENT, "bad argument");
        SB_REQUIRE(r <= (int64_t)1 << 20, SB_ERR_INVALID_ARGUMENT, "apply_block_tensor: too many vectors");
        Operator& o = *op->op;
        SB_CUDA(cudaSetDevice(o.device));
        maybe_inject(SB_INJECT_LAUNCH);
        tensor_block_product(o, reinterpret_cast<const float2*>(x_dev), o.n, static_cast<int>(r),
                             reinterpret_cast<float2*>(y_dev), o.n, o.stream);
        SB_CUDA(cudaStreamSynchronize(o.stream));
        SB_REQUIRE(tensor_status(o, true) == 0, SB_ERR_DEVICE_CHECK,
                   "apply_block_tensor: a pipeline wait of the tensor-core kernel timed out");
    });
}

SB_API int sb_operator_block_residual(const sb_operator* op, const sb_complex* b, const sb_complex* x, int64_t r,
                                      sb_complex* res) {
    return guarded([&] {
        SB_REQUIRE(op && op->op && b && x && res && r >= 1, SB_ERR_INVALID_ARGUMENT, "bad argument");
        SB_REQUIRE(r <= 65536, SB_ERR_INVALID_ARGUMENT, "block_residual: at most 65536 vectors");
        Operator& o = *op->op;
        SB_REQUIRE(o.A64.p, SB_ERR_INVALID_ARGUMENT,
                   "block_residual: needs the complex128 matrix (SB_PRECISION_FP64 or SB_PRECISION_FP64_FP32)");
        const int64_t n = o.n;
        SB_CUDA(cudaSetDevice(o.device));
        maybe_inject(SB_INJECT_LAUNCH);
        // n x r row-major blocks (the reference's DenseMatrix layout) <-> vector-major device copies
        std::vector<sb_complex> t(n * r), u(n * r);
        DevBuf db, dx, dr;
        db.alloc(sizeof(double2) * n * r);
        dx.alloc(sizeof(double2) * n * r);
        dr.alloc(sizeof(double2) * n * r);
        for (int64_t i = 0; i < n; ++i)
            for (int64_t c = 0; c < r; ++c) {
                t[c * n + i] = b[i * r + c];
                u[c * n + i] = x[i * r + c];
            }
        SB_CUDA(cudaMemcpyAsync(db.p, t.data(), sizeof(double2) * n * r, cudaMemcpyHostToDevice, o.stream));
        SB_CUDA(cudaMemcpyAsync(dx.p, u.data(), sizeof(double2) * n * r, cudaMemcpyHostToDevice, o.stream));
        ozaki_residual(o, db.as<double2>(), n, dx.as<double2>(), n, static_cast<int>(r), dr.as<double2>(), n, o.stream);
        SB_CUDA(cudaMemcpyAsync(t.data(), dr.p, sizeof(double2) * n * r, cudaMemcpyDeviceToHost, o.stream));
        SB_CUDA(cudaStreamSynchronize(o.stream));
        SB_REQUIRE(ozaki_status(o, true) == 0, SB_ERR_DEVICE_CHECK,
                   "block_residual: a pipeline wait of the block-residual kernel timed out");
        for (int64_t i = 0; i < n; ++i)
            for (int64_t c = 0; c < r; ++c) res[i * r + c] = t[c * n + i];
    });
}

SB_API int sb_operator_block_residual_device(const sb_operator* op, const sb_complex* b_dev, const sb_complex* x_dev,
                                             int64_t r, sb_complex* res_dev) {
    return guarded([&] {
        SB_REQUIRE(op && op->op && b_dev && x_dev && res_dev && r >= 1, SB_ERR_INVALID_ARGUMENT, "bad argument");
        SB_REQUIRE(r <= 65536, SB_ERR_INVALID_ARGUMENT, "block_residual: at most 65536 vectors");
        Operator& o = *op->op;
        SB_REQUIRE(o.A64.p, SB_ERR_INVALID_ARGUMENT,
                   "block_residual: needs the complex128 matrix (SB_PRECISION_FP64 or SB_PRECISION_FP64_FP32)");
        SB_CUDA(cudaSetDevice(o.device));
        maybe_inject(SB_INJECT_LAUNCH);
        ozaki_residual(o, reinterpret_cast<const double2*>(b_dev), o.n, reinterpret_cast<const double2*>(x_dev), o.n,
                       static_cast<int>(r), reinterpret_cast<double2*>(res_dev), o.n, o.stream);
        SB_CUDA(cudaStreamSynchronize(o.stream));
        SB_REQUIRE(ozaki_status(o, true) == 0, SB_ERR_DEVICE_CHECK,
                   "block_residual: a pipeline wait of the block-residual kernel timed out");
    });
}

SB_API int sb_gmres_multi(const sb_operator* op, const sb_complex* b, int64_t r, const sb_ir_config* cfg,
                          sb_complex* x, sb_gmres_stats* stats) {
    return guarded([&] {
        SB_REQUIRE(op && op->op && b && x && cfg && stats && r >= 1, SB_ERR_INVALID_ARGUMENT, "bad argument");
        SB_REQUIRE(r <= 65536, SB_ERR_INVALID_ARGUMENT, "gmres_multi: at most 65536 right-hand sides");
        check_ir(cfg);
        Operator& o = *op->op;
        const int64_t n = o.n;
        SB_REQUIRE(all_finite(b, n * r), SB_ERR_NOT_FINITE, "gmres_multi: non-finite right-hand side block");
        SB_CUDA(cudaSetDevice(o.device));
        maybe_inject(SB_INJECT_LAUNCH);
        // n x r row-major block (the reference's DenseMatrix layout) <-> right-hand-side-major device
        std::vector<sb_complex> t(n * r);
        for (int64_t i = 0; i < n; ++i)
            for (int64_t c = 0; c < r; ++c) t[c * n + i] = b[i * r + c];
        DevBuf db, dx;
        db.alloc(sizeof(double2) * n * r);
        dx.alloc(sizeof(double2) * n * r);
        h2d_sync(db.p, t.data(), sizeof(double2) * n * r);
        multi_solve_device(o, db.as<double2>(), n, static_cast<int>(r), dx.as<double2>(), n, *cfg, stats);
        SB_CUDA(cudaMemcpy(t.data(), dx.p, sizeof(double2) * n * r, cudaMemcpyDeviceToHost));
        for (int64_t i = 0; i < n; ++i)
            for (int64_t c = 0; c < r; ++c) x[i * r + c] = t[c * n + i];
    });
}

SB_API int sb_gmres_multi_device(const sb_operator* op, const sb_complex* b_dev, int64_t r, const sb_ir_config* cfg,
                                 sb_complex* x_dev, sb_gmres_stats* stats) {
    return guarded([&] {
        SB_REQUIRE(op && op->op && b_dev && x_dev && cfg && stats && r >= 1, SB_ERR_INVALID_ARGUMENT, "bad argument");
        SB_REQUIRE(r <= 65536, SB_ERR_INVALID_ARGUMENT, "gmres_multi: at most 65536 right-hand sides");
        check_ir(cfg);
        Operator& o = *op->op;
        maybe_inject(SB_INJECT_LAUNCH);
        multi_solve_device(o, reinterpret_cast<const double2*>(b_dev), o.n, static_cast<int>(r),
                           reinterpret_cast<double2*>(x_dev), o.n, *cfg, stats);
    });
}

// Preconditioners of the FP64 GMRES: identity, Jacobi (left) or block-Jacobi (right, needs the
// complex128 matrix).
static void check_gmres_precond(const Operator& o, int precond) {
    SB_REQUIRE(precond == SB_PRECOND_IDENTITY || precond == SB_PRECOND_JACOBI || precond == SB_PRECOND_BLOCK_JACOBI,
               SB_ERR_INVALID_ARGUMENT, "unknown preconditioner");
    if (precond == SB_PRECOND_BLOCK_JACOBI)
        SB_REQUIRE(o.A64.p, SB_ERR_INVALID_ARGUMENT,
                   "SB_PRECOND_BLOCK_JACOBI needs the complex128 matrix (SB_PRECISION_FP64 or SB_PRECISION_FP64_FP32)");
}

SB_API int sb_preconditioner_apply(const sb_operator* op, int precond, const sb_complex* x, sb_complex* y) {
    return guarded([&] {
        SB_REQUIRE(op && op->op && x && y, SB_ERR_INVALID_ARGUMENT, "null argument");
        Operator& o = *op->op;
        check_gmres_precond(o, precond);
        if (precond == SB_PRECOND_IDENTITY) {
            std::memcpy(y, x, sizeof(sb_complex) * o.n);
            return;
        }
        SB_CUDA(cudaSetDevice(o.device));
        DevBuf dx, dy;
        dx.alloc(sizeof(double2) * o.n);
        SB_CUDA(cudaMemcpyAsync(dx.p, x, sizeof(double2) * o.n, cudaMemcpyHostToDevice, o.stream));
        if (precond == SB_PRECOND_BLOCK_JACOBI) {
            bj64_prepare(o);
            dy.alloc(sizeof(double2) * o.n);
            bj64_apply(o, dx.as<double2>(), dy.as<double2>(), Gate{});
            SB_CUDA(cudaMemcpyAsync(dx.p, dy.p, sizeof(double2) * o.n, cudaMemcpyDeviceToDevice, o.stream));
        } else {
            jacobi_apply<double2>(o.diag.as<double2>(), dx.as<double2>(), dx.as<double2>(), o.n, o.stream);
        }
        SB_CUDA(cudaMemcpyAsync(y, dx.p, sizeof(double2) * o.n, cudaMemcpyDeviceToHost, o.stream));
        SB_CUDA(cudaStreamSynchronize(o.stream));
    });
}

SB_API int sb_rhs_plane_wave(const sb_mesh* mesh, const sb_physics* physics, sb_complex beta, const double* dirs,
                             const sb_complex* amps, int64_t r, sb_complex* rhs) {
    return guarded([&] {
        SB_REQUIRE(mesh && mesh->m && physics && dirs && rhs && r >= 1, SB_ERR_INVALID_ARGUMENT, "bad argument");
        SB_REQUIRE(sb_physics_validate(physics) == SB_OK, SB_ERR_INVALID_ARGUMENT, "invalid physics: " + t_err);
        check_beta(beta);
        for (int64_t q = 0; q < 3 * r; ++q)
            SB_REQUIRE(std::isfinite(dirs[q]), SB_ERR_INVALID_ARGUMENT, "non-finite direction");
        const Mesh& m = *mesh->m;
        SB_CUDA(cudaSetDevice(m.device));
        DevBuf d;
        d.alloc(sizeof(double2) * m.n * r);
        incident_plane_wave(m, *physics, beta.re, beta.im, dirs, reinterpret_cast<const double*>(amps), r,
                            d.as<double2>(), 0, false);
        SB_CUDA(cudaMemcpy(rhs, d.p, sizeof(double2) * m.n * r, cudaMemcpyDeviceToHost));
    });
}

SB_API int sb_field_eval(const sb_mesh* mesh, const sb_physics* physics, const sb_complex* surface_pressure,
                         const sb_complex* surface_velocity, const double* points, int64_t m, sb_complex* field) {
    return guarded([&] {
        SB_REQUIRE(mesh && mesh->m && physics && surface_pressure && m >= 0, SB_ERR_INVALID_ARGUMENT,
                   "bad argument");
        SB_REQUIRE(m == 0 || (points && field), SB_ERR_INVALID_ARGUMENT, "null points or output");
        SB_REQUIRE(sb_physics_validate(physics) == SB_OK, SB_ERR_INVALID_ARGUMENT, "invalid physics: " + t_err);
        const Mesh& me = *mesh->m;
        SB_REQUIRE(!me.quad, SB_ERR_UNSUPPORTED_ELEMENT, "field_eval: Tri3 meshes only");
        SB_REQUIRE(all_finite(surface_pressure, me.n), SB_ERR_NOT_FINITE, "field_eval: non-finite surface pressure");
        if (surface_velocity)
            SB_REQUIRE(all_finite(surface_velocity, me.n), SB_ERR_NOT_FINITE,
                       "field_eval: non-finite surface velocity");
        for (int64_t q = 0; q < 3 * m; ++q)
            SB_REQUIRE(std::isfinite(points[q]), SB_ERR_INVALID_ARGUMENT, "field_eval: non-finite point");
        if (m == 0) return;
        SB_CUDA(cudaSetDevice(me.device));
        maybe_inject(SB_INJECT_LAUNCH);
        DevBuf dp, dv, dx, dout;
        dp.alloc(sizeof(double2) * me.n);
        h2d_sync(dp.p, surface_pressure, sizeof(double2) * me.n);
        if (surface_velocity) {
            dv.alloc(sizeof(double2) * me.n);
            h2d_sync(dv.p, surface_velocity, sizeof(double2) * me.n);
        }
        dx.alloc(sizeof(double) * 3 * m);
        dout.alloc(sizeof(double2) * m);
        h2d_sync(dx.p, points, sizeof(double) * 3 * m);
        field_eval(me, *physics, dp.as<double2>(), surface_velocity ? dv.as<double2>() : nullptr, dx.as<double>(), m,
                   dout.as<double2>(), 0);
        SB_CUDA(cudaMemcpy(field, dout.p, sizeof(double2) * m, cudaMemcpyDeviceToHost));
        SB_REQUIRE(all_finite(field, m), SB_ERR_NOT_FINITE, "field_eval: non-finite result (point on the surface?)");
    });
}

static void check_cfg(const sb_gmres_config* cfg) {
    SB_REQUIRE(cfg, SB_ERR_INVALID_ARGUMENT, "null config");
    SB_REQUIRE(cfg->max_iterations > 0 && cfg->restart > 0, SB_ERR_INVALID_ARGUMENT,
               "max_iterations and restart must be positive");
    SB_REQUIRE(cfg->restart <= 120, SB_ERR_INVALID_ARGUMENT, "restart must be <= 120");
    SB_REQUIRE(std::isfinite(cfg->tolerance) && cfg->tolerance > 0, SB_ERR_INVALID_ARGUMENT,
               "tolerance must be finite and positive");
}

SB_API int sb_gmres_device(const sb_operator* op, const sb_complex* b_dev, sb_complex* x_dev, int x0_given,
                           const sb_gmres_config* cfg, int precond, sb_gmres_stats* stats) {
    return guarded([&] {
        SB_REQUIRE(op && op->op && b_dev && x_dev && stats, SB_ERR_INVALID_ARGUMENT, "null argument");
        check_cfg(cfg);
        check_gmres_precond(*op->op, precond);
        maybe_inject(SB_INJECT_LAUNCH);
        gmres_fp64(*op->op, reinterpret_cast<const double2*>(b_dev), reinterpret_cast<double2*>(x_dev), x0_given != 0,
                   *cfg, precond, *stats);
    });
}

SB_API int sb_gmres(const sb_operator* op, const sb_complex* b, const sb_complex* x0, const sb_gmres_config* cfg,
                    int precond, sb_complex* x, sb_gmres_stats* stats) {
    return guarded([&] {
        SB_REQUIRE(op && op->op && b && x && stats, SB_ERR_INVALID_ARGUMENT, "null argument");
        check_cfg(cfg);
        const Operator& o = *op->op;
        SB_REQUIRE(all_finite(b, o.n), SB_ERR_NOT_FINITE, "gmres: non-finite right-hand side");
        if (x0) SB_REQUIRE(all_finite(x0, o.n), SB_ERR_NOT_FINITE, "gmres: non-finite initial guess");
        SB_CUDA(cudaSetDevice(o.device));
        DevBuf db, dx;
        db.alloc(sizeof(double2) * o.n);
        dx.alloc(sizeof(double2) * o.n);
        SB_CUDA(cudaMemcpyAsync(db.p, b, sizeof(double2) * o.n, cudaMemcpyHostToDevice, o.stream));
        if (x0) SB_CUDA(cudaMemcpyAsync(dx.p, x0, sizeof(double2) * o.n, cudaMemcpyHostToDevice, o.stream));
        check_gmres_precond(o, precond);
        maybe_inject(SB_INJECT_LAUNCH);
        gmres_fp64(o, db.as<double2>(), dx.as<double2>(), x0 != nullptr, *cfg, precond, *stats);
        SB_CUDA(cudaMemcpyAsync(x, dx.p, sizeof(double2) * o.n, cudaMemcpyDeviceToHost, o.stream));
        SB_CUDA(cudaStreamSynchronize(o.stream));
    });
}

static void check_ir(const sb_ir_config* cfg) {
    SB_REQUIRE(cfg, SB_ERR_INVALID_ARGUMENT, "null config");
    SB_REQUIRE(cfg->max_refinements > 0 && cfg->inner_restart > 0 && cfg->inner_max_iterations > 0,
               SB_ERR_INVALID_ARGUMENT, "iteration limits must be positive");
    SB_REQUIRE(cfg->inner_restart <= 120, SB_ERR_INVALID_ARGUMENT, "inner_restart must be <= 120");
    SB_REQUIRE(std::isfinite(cfg->tolerance) && cfg->tolerance > 0 && std::isfinite(cfg->inner_tolerance) &&
                   cfg->inner_tolerance > 0,
               SB_ERR_INVALID_ARGUMENT, "tolerances must be finite and positive");
}

SB_API int sb_gmres_mixed_device(const sb_operator* op, const sb_complex* b_dev, sb_complex* x_dev, int x0_given,
                                 const sb_ir_config* cfg, sb_gmres_stats* stats) {
    return guarded([&] {
        SB_REQUIRE(op && op->op && b_dev && x_dev && stats, SB_ERR_INVALID_ARGUMENT, "null argument");
        check_ir(cfg);
        maybe_inject(SB_INJECT_LAUNCH);
        gmres_mixed_ir(*op->op, reinterpret_cast<const double2*>(b_dev), reinterpret_cast<double2*>(x_dev),
                       x0_given != 0, *cfg, *stats);
    });
}

SB_API int sb_gmres_mixed(const sb_operator* op, const sb_complex* b, const sb_complex* x0, const sb_ir_config* cfg,
                          sb_complex* x, sb_gmres_stats* stats) {
    return guarded([&] {
        SB_REQUIRE(op && op->op && b && x && stats, SB_ERR_INVALID_ARGUMENT, "null argument");
        check_ir(cfg);
        const Operator& o = *op->op;
        SB_REQUIRE(all_finite(b, o.n), SB_ERR_NOT_FINITE, "gmres: non-finite right-hand side");
        if (x0) SB_REQUIRE(all_finite(x0, o.n), SB_ERR_NOT_FINITE, "gmres: non-finite initial guess");
        SB_CUDA(cudaSetDevice(o.device));
        DevBuf db, dx;
        db.alloc(sizeof(double2) * o.n);
        dx.alloc(sizeof(double2) * o.n);
        SB_CUDA(cudaMemcpyAsync(db.p, b, sizeof(double2) * o.n, cudaMemcpyHostToDevice, o.stream));
        if (x0) SB_CUDA(cudaMemcpyAsync(dx.p, x0, sizeof(double2) * o.n, cudaMemcpyHostToDevice, o.stream));
        maybe_inject(SB_INJECT_LAUNCH);
        gmres_mixed_ir(o, db.as<double2>(), dx.as<double2>(), x0 != nullptr, *cfg, *stats);
        SB_CUDA(cudaMemcpyAsync(x, dx.p, sizeof(double2) * o.n, cudaMemcpyDeviceToHost, o.stream));
        SB_CUDA(cudaStreamSynchronize(o.stream));
    });
}

SB_API int sb_operator_set_inner_precision(sb_operator* op, int inner) {
    return guarded([&] {
        SB_REQUIRE(op && op->op, SB_ERR_INVALID_ARGUMENT, "null argument");
        SB_REQUIRE(inner == SB_INNER_FP32 || inner == SB_INNER_FP16, SB_ERR_INVALID_ARGUMENT,
                   "inner precision must be SB_INNER_FP32 or SB_INNER_FP16");
        SB_REQUIRE(inner == SB_INNER_FP32 || op->op->A32.p, SB_ERR_INVALID_ARGUMENT,
                   "SB_INNER_FP16 needs a complex64 matrix (SB_PRECISION_FP64_FP32 or SB_PRECISION_FP32)");
        op->op->inner = inner;
        if (inner == SB_INNER_FP32) {
            op->op->A16.release();
            op->op->half_valid = false;
            op->op->half_check = false;
        }
    });
}

SB_API int sb_operator_set_inner_preconditioner(sb_operator* op, int kind, int block_size) {
    return guarded([&] {
        SB_REQUIRE(op && op->op, SB_ERR_INVALID_ARGUMENT, "null argument");
        SB_REQUIRE(kind == SB_INNER_PRECOND_NONE || kind == SB_INNER_PRECOND_BLOCK_JACOBI, SB_ERR_INVALID_ARGUMENT,
                   "inner preconditioner must be SB_INNER_PRECOND_NONE or SB_INNER_PRECOND_BLOCK_JACOBI");
        Operator& o = *op->op;
        if (kind == SB_INNER_PRECOND_BLOCK_JACOBI) {
            SB_REQUIRE(block_size == 32 || block_size == 64 || block_size == 96 || block_size == 128,
                       SB_ERR_INVALID_ARGUMENT, "block_size must be 32, 64, 96 or 128");
            SB_REQUIRE(o.A32.p, SB_ERR_INVALID_ARGUMENT,
                       "the block-Jacobi inner preconditioner needs a complex64 matrix (SB_PRECISION_FP64_FP32 or "
                       "SB_PRECISION_FP32)");
            if (block_size != o.bj_size) o.bj_valid = o.bj64_valid = false;
            o.bj_size = block_size;
        } else {
            o.bj_inv.release();
            o.bj_valid = false;
        }
        o.inner_precond = kind;
    });
}

SB_API int sb_operator_set_block_jacobi_size(sb_operator* op, int block_size) {
    return guarded([&] {
        SB_REQUIRE(op && op->op, SB_ERR_INVALID_ARGUMENT, "null argument");
        SB_REQUIRE(block_size == 32 || block_size == 64 || block_size == 96 || block_size == 128,
                   SB_ERR_INVALID_ARGUMENT, "block_size must be 32, 64, 96 or 128");
        Operator& o = *op->op;
        if (block_size != o.bj_size) o.bj_valid = o.bj64_valid = false;
        o.bj_size = block_size;
    });
}

SB_API int sb_rhs_plane_wave_device(const sb_operator* op, const double* dirs, const sb_complex* amps, int64_t r,
                                    sb_complex* rhs_dev) {
    return guarded([&] {
        SB_REQUIRE(op && op->op && dirs && rhs_dev && r >= 1, SB_ERR_INVALID_ARGUMENT, "bad argument");
        for (int64_t q = 0; q < 3 * r; ++q)
            SB_REQUIRE(std::isfinite(dirs[q]), SB_ERR_INVALID_ARGUMENT, "non-finite direction");
        const Operator& o = *op->op;
        SB_REQUIRE(o.mesh, SB_ERR_INVALID_ARGUMENT, "operator was not assembled from a mesh");
        if (o.basis != SB_BASIS_CONSTANT) {
            incident_plane_wave_at(o.device, o.lin_cp.as<double>(), o.lin_cn.as<double>(), o.n, o.n, o.phys, o.beta_re,
                                   o.beta_im, dirs, reinterpret_cast<const double*>(amps), r,
                                   reinterpret_cast<double2*>(rhs_dev), o.stream);
            return;
        }
        incident_plane_wave(*o.mesh, o.phys, o.beta_re, o.beta_im, dirs, reinterpret_cast<const double*>(amps), r,
                            reinterpret_cast<double2*>(rhs_dev), o.stream, false);
    });
}

// ---- GCRO-DR ----
SB_API int sb_gcro_subspace_create(int device, int64_t k, sb_gcro_subspace** out) {
    return guarded([&] {
        SB_REQUIRE(out, SB_ERR_INVALID_ARGUMENT, "null argument");
        *out = nullptr;
        SB_REQUIRE(k >= 0 && k <= 100, SB_ERR_INVALID_ARGUMENT, "recycled subspace size must be in 0..100");
        int count = 0;
        SB_CUDA(cudaGetDeviceCount(&count));
        SB_REQUIRE(device >= 0 && device < count, SB_ERR_INVALID_ARGUMENT, "no such device");
        *out = new sb_gcro_subspace{recycle_create(device, k)};
    });
}

SB_API int sb_gcro_subspace_destroy(sb_gcro_subspace* s) {
    return guarded([&] {
        if (!s) return;
        recycle_destroy(s->s);
        delete s;
    });
}

SB_API int sb_gcro_subspace_reset(sb_gcro_subspace* s) {
    return guarded([&] {
        SB_REQUIRE(s && s->s, SB_ERR_INVALID_ARGUMENT, "null subspace");
        recycle_reset(*s->s);
    });
}

SB_API int sb_gcro_subspace_info(const sb_gcro_subspace* s, int64_t* num_vectors, int64_t* target, int64_t* n) {
    return guarded([&] {
        SB_REQUIRE(s && s->s, SB_ERR_INVALID_ARGUMENT, "null subspace");
        recycle_info(*s->s, num_vectors, target, n);
    });
}

SB_API int sb_gcro_subspace_get_vectors(const sb_gcro_subspace* s, sb_complex* u) {
    return guarded([&] {
        SB_REQUIRE(s && s->s && u, SB_ERR_INVALID_ARGUMENT, "null argument");
        recycle_get(*s->s, reinterpret_cast<double2*>(u));
    });
}

SB_API int sb_gcro_subspace_set_vectors(sb_gcro_subspace* s, int64_t count, int64_t n, const sb_complex* u) {
    return guarded([&] {
        SB_REQUIRE(s && s->s && (u || count == 0), SB_ERR_INVALID_ARGUMENT, "null argument");
        if (count > 0) {
            SB_REQUIRE(n > 0, SB_ERR_INVALID_ARGUMENT, "vector length must be positive");
            SB_REQUIRE(all_finite(u, count * n), SB_ERR_NOT_FINITE, "recycled subspace: non-finite vector entry");
        }
        recycle_set(*s->s, count, n, reinterpret_cast<const double2*>(u));
    });
}

SB_API int sb_gcro_dr_device(const sb_operator* op, const sb_complex* b_dev, sb_complex* x_dev, int x0_given,
                             sb_gcro_subspace* s, const sb_gmres_config* cfg, int precond, sb_gmres_stats* stats) {
    return guarded([&] {
        SB_REQUIRE(op && op->op && s && s->s && b_dev && x_dev && stats, SB_ERR_INVALID_ARGUMENT, "null argument");
        check_cfg(cfg);
        SB_REQUIRE(precond == SB_PRECOND_IDENTITY || precond == SB_PRECOND_JACOBI, SB_ERR_INVALID_ARGUMENT,
                   "unknown preconditioner");
        maybe_inject(SB_INJECT_LAUNCH);
        gcro_dr(*op->op, reinterpret_cast<const double2*>(b_dev), reinterpret_cast<double2*>(x_dev), x0_given != 0,
                *s->s, *cfg, precond, *stats);
    });
}

SB_API int sb_gcro_dr(const sb_operator* op, const sb_complex* b, const sb_complex* x0, sb_gcro_subspace* s,
                      const sb_gmres_config* cfg, int precond, sb_complex* x, sb_gmres_stats* stats) {
    return guarded([&] {
        SB_REQUIRE(op && op->op && s && s->s && b && x && stats, SB_ERR_INVALID_ARGUMENT, "null argument");
        check_cfg(cfg);
        SB_REQUIRE(precond == SB_PRECOND_IDENTITY || precond == SB_PRECOND_JACOBI, SB_ERR_INVALID_ARGUMENT,
                   "unknown preconditioner");
        const Operator& o = *op->op;
        SB_REQUIRE(all_finite(b, o.n), SB_ERR_NOT_FINITE, "gcro_dr: non-finite right-hand side");
        if (x0) SB_REQUIRE(all_finite(x0, o.n), SB_ERR_NOT_FINITE, "gcro_dr: non-finite initial guess");
        SB_CUDA(cudaSetDevice(o.device));
        DevBuf db, dx;
        db.alloc(sizeof(double2) * o.n);
        dx.alloc(sizeof(double2) * o.n);
        SB_CUDA(cudaMemcpyAsync(db.p, b, sizeof(double2) * o.n, cudaMemcpyHostToDevice, o.stream));
        if (x0) SB_CUDA(cudaMemcpyAsync(dx.p, x0, sizeof(double2) * o.n, cudaMemcpyHostToDevice, o.stream));
        maybe_inject(SB_INJECT_LAUNCH);
        gcro_dr(o, db.as<double2>(), dx.as<double2>(), x0 != nullptr, *s->s, *cfg, precond, *stats);
        SB_CUDA(cudaMemcpyAsync(x, dx.p, sizeof(double2) * o.n, cudaMemcpyDeviceToHost, o.stream));
        SB_CUDA(cudaStreamSynchronize(o.stream));
    });
}

SB_API int sb_memory_trim(int device) {
    return guarded([&] {
        solve_work_pool_trim(device);
        memory_trim(device);
    });
}

SB_API int sb_memory_stats(int device, int64_t* in_use_bytes, int64_t* cached_bytes) {
    return guarded([&] { memory_stats(device, in_use_bytes, cached_bytes); });
}

SB_API int sb_profile_enable(int on) {
    return guarded([&] {
        g_prof_on = on != 0;
        g_prof_mask = ~0u;
    });
}

SB_API int sb_profile_enable_classes(unsigned mask) {
    return guarded([&] {
        g_prof_on = mask != 0;
        g_prof_mask = mask;
    });
}

SB_API int sb_profile_read(sb_profile* out, int reset) {
    return guarded([&] {
        SB_REQUIRE(out, SB_ERR_INVALID_ARGUMENT, "null output");
        profile_read(out, reset != 0);
    });
}

SB_API int sb_event_create(void** event) {
    return guarded([&] {
        SB_REQUIRE(event, SB_ERR_INVALID_ARGUMENT, "null output");
        cudaEvent_t e;
        SB_CUDA(cudaEventCreate(&e));
        *event = e;
    });
}

SB_API int sb_event_destroy(void* event) {
    return guarded([&] {
        if (event) SB_CUDA(cudaEventDestroy(static_cast<cudaEvent_t>(event)));
    });
}

SB_API int sb_event_record(void* event, const sb_operator* op) {
    return guarded([&] {
        SB_REQUIRE(event && op && op->op, SB_ERR_INVALID_ARGUMENT, "null argument");
        SB_CUDA(cudaSetDevice(op->op->device));
        SB_CUDA(cudaEventRecord(static_cast<cudaEvent_t>(event), op->op->stream));
    });
}

SB_API int sb_event_elapsed_ms(void* start, void* stop, float* ms) {
    return guarded([&] {
        SB_REQUIRE(start && stop && ms, SB_ERR_INVALID_ARGUMENT, "null argument");
        SB_CUDA(cudaEventSynchronize(static_cast<cudaEvent_t>(stop)));
        SB_CUDA(cudaEventElapsedTime(ms, static_cast<cudaEvent_t>(start), static_cast<cudaEvent_t>(stop)));
    });
}

SB_API int sb_math_sincos(int device, const double* x, int64_t n, double* s, double* c) {
    return guarded([&] {
        SB_REQUIRE(x && s && c && n >= 1, SB_ERR_INVALID_ARGUMENT, "bad argument");
        int ndev = 0;
        SB_CUDA(cudaGetDeviceCount(&ndev));
        SB_REQUIRE(device >= 0 && device < ndev, SB_ERR_CUDA, "CUDA device not available");
        device_sincos(device, x, n, s, c);
    });
}

SB_API int sb_inject_failure(int point) {
    return guarded([&] {
        SB_REQUIRE(point == SB_INJECT_NONE || point == SB_INJECT_ALLOC || point == SB_INJECT_LAUNCH,
                   SB_ERR_INVALID_ARGUMENT, "unknown injection point");
        std::lock_guard<std::mutex> lock(g_inject_mu);
        g_inject_point = point;
    });
}

}  // extern "C"
