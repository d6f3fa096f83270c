// Exterior field evaluation from constant Tri3 surface data: the scattered pressure at arbitrary
// points off the surface, the step after the solve.
//
// Reference: compute_scattered_field_checked / compute_scattered_field (crates/sonium-bem/src/core/
// postprocess/pressure.rs:250-289, 868-894) -> compute_scattered_field_with_incident (:1388-1448)
// with explicit surface velocity (constant_cauchy_data, :1489-1491) -> integrate_element_field
// (:1566-1606: Tri3 with the 7-point rule of triangle_quadrature(3)) -> integrate_quad_point
// (:1987-2042):
//   p_scat(x) = sum_e sum_q [ p_e (e^{ikr} / 4 pi r)(-1/r + ik)((y_q - x).n_y / r)
//                             - v_e (i pressure_factor)(e^{ikr} / 4 pi r) ] J_e w_q.
// The reference's CUDA kernel for it (bem_kernels.cu:701-813) is one thread per (point, element)
// with host-built charts; here one thread owns an evaluation point and sweeps a range of elements
// whose 7 quadrature points per element are staged in shared memory by the CTA (computed from the
// element records once per CTA, reused by 128 points), with FP64 arithmetic throughout. The
// element range is split over grid.y so small point sets still fill the GPU; the per-range partial
// sums are added in a fixed order by a second kernel (deterministic results).

#include "sb_device.cuh"
#include "sb_internal.cuh"
#include "sb_profile.cuh"

struct sb_mesh {
    sb::Mesh* m;
};

namespace sb {
namespace {

constexpr int kFieldPoints = 128;  // evaluation points per CTA (one per thread)
constexpr int kFieldElems = 32;    // elements staged per shared-memory tile
constexpr int kTR7 = 7;

// The 7-point degree-5 rule on the unit simplex (the reference's GAUCORWEI_TR7 table, gauss.rs:
// 516-524, weights summing to 1); triangle_quadrature scales the weights by the reference-triangle
// area 0.5.
__constant__ double c_tr7[kTR7][3] = {{0.333333333333333, 0.333333333333333, 0.225},
                                      {0.797426985353087, 0.101286507323456, 0.125939180544827},
                                      {0.101286507323456, 0.797426985353087, 0.125939180544827},
                                      {0.101286507323456, 0.101286507323456, 0.125939180544827},
                                      {0.470142064105115, 0.059715871789770, 0.132394152788506},
                                      {0.059715871789770, 0.470142064105115, 0.132394152788506},
                                      {0.470142064105115, 0.470142064105115, 0.132394152788506}};

int64_t cdiv(int64_t a, int64_t b) { return (a + b - 1) / b; }

#define EL(f, e) elem[(int64_t)(f) * ld + (e)]

// partial[chunk * m + i] = contribution of elements [chunk * per, (chunk + 1) * per) at point i.
__global__ void __launch_bounds__(kFieldPoints) k_field(const double* __restrict__ elem, int64_t n, int64_t ld,
                                                        const double2* __restrict__ pressure,
                                                        const double2* __restrict__ velocity, double wavruim,
                                                        double pressure_factor, const double* __restrict__ points,
                                                        int64_t m, int64_t per, double2* __restrict__ partial) {
    __shared__ double sq[kFieldElems * kTR7][3];  // quadrature points
    __shared__ double sw[kFieldElems * kTR7];     // J w_q
    __shared__ double sn[kFieldElems][3];         // unit normal
    __shared__ double2 sp[kFieldElems], sv[kFieldElems];
    const int64_t i = blockIdx.x * (int64_t)kFieldPoints + threadIdx.x;
    const int64_t e0 = blockIdx.y * per;
    const int64_t e1 = (e0 + per < n) ? e0 + per : n;
    double x0 = 0.0, x1 = 0.0, x2 = 0.0;
    if (i < m) {
        x0 = points[3 * i];
        x1 = points[3 * i + 1];
        x2 = points[3 * i + 2];
    }
    double2 acc = make_double2(0.0, 0.0);
    for (int64_t t0 = e0; t0 < e1; t0 += kFieldElems) {
        const int cnt = static_cast<int>((e1 - t0) < kFieldElems ? (e1 - t0) : kFieldElems);
        __syncthreads();  // the previous tile is no longer read
        for (int s = threadIdx.x; s < cnt * kTR7; s += kFieldPoints) {
            const int le = s / kTR7, q = s % kTR7;
            const int64_t e = t0 + le;
            const double xi = c_tr7[q][0], eta = c_tr7[q][1];
            const double sf[3] = {1.0 - xi - eta, xi, eta};
            // position = sum_a N_a v_a in the order quadrature_geometry accumulates it
            for (int d = 0; d < 3; ++d) {
                double p = 0.0;
                for (int a = 0; a < 3; ++a) p = __dadd_rn(p, __dmul_rn(sf[a], EL(EV0X + 3 * a + d, e)));
                sq[s][d] = p;
            }
            sw[s] = __dmul_rn(EL(EJAC, e), __dmul_rn(c_tr7[q][2], 0.5));
        }
        for (int le = threadIdx.x; le < cnt; le += kFieldPoints) {
            const int64_t e = t0 + le;
            sn[le][0] = EL(ENX, e);
            sn[le][1] = EL(ENY, e);
            sn[le][2] = EL(ENZ, e);
            sp[le] = pressure[e];
            sv[le] = velocity ? velocity[e] : make_double2(0.0, 0.0);
        }
        __syncthreads();
        if (i >= m) continue;
        for (int le = 0; le < cnt; ++le) {
            const double2 p = sp[le], v = sv[le];
            const bool with_v = hypot(v.x, v.y) > 1e-15;
            for (int q = 0; q < kTR7; ++q) {
                const int s = le * kTR7 + q;
                const double r0 = sq[s][0] - x0, r1 = sq[s][1] - x1, r2 = sq[s][2] - x2;
                const double r = sqrt(r0 * r0 + r1 * r1 + r2 * r2);
                if (r < 1e-15) continue;
                double sk, ck;
                sb_sincos(wavruim * r, &sk, &ck);
                const double inv = 1.0 / (4.0 * 3.14159265358979323846 * r);
                const double gr = ck * inv, gi = sk * inv;              // e^{ikr} / (4 pi r)
                const double ir = -1.0 / r;                             // (-1/r + i k)
                const double zr = gr * ir - gi * wavruim, zi = gr * wavruim + gi * ir;
                const double drdn = (r0 * sn[le][0] + r1 * sn[le][1] + r2 * sn[le][2]) / r;
                const double wj = sw[s];
                const double dr = zr * drdn, di = zi * drdn;
                acc.x += (p.x * dr - p.y * di) * wj;
                acc.y += (p.x * di + p.y * dr) * wj;
                if (with_v) {
                    // - v (i pf) G J w
                    const double vr = -v.y * pressure_factor, vi = v.x * pressure_factor;
                    acc.x -= (vr * gr - vi * gi) * wj;
                    acc.y -= (vr * gi + vi * gr) * wj;
                }
            }
        }
    }
    if (i < m) partial[blockIdx.y * m + i] = acc;
}

// out[i] = sum over the element ranges, in order.
__global__ void k_field_sum(const double2* __restrict__ partial, int64_t m, int chunks, double2* __restrict__ out) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= m) return;
    double2 s = make_double2(0.0, 0.0);
    for (int c = 0; c < chunks; ++c) {
        const double2 v = partial[(int64_t)c * m + i];
        s.x += v.x;
        s.y += v.y;
    }
    out[i] = s;
}

}  // namespace

void field_eval(const Mesh& mesh, const sb_physics& ph, const double2* pressure, const double2* velocity,
                const double* points, int64_t m, double2* out, cudaStream_t s) {
    const int64_t tiles = cdiv(m, kFieldPoints);
    // enough CTAs to fill the GPU twice over, each on a range of whole element tiles
    const int64_t want = 2 * device_sm_count(mesh.device);
    int64_t chunks = tiles >= want ? 1 : cdiv(want, tiles);
    int64_t per = cdiv(cdiv(mesh.n, chunks), kFieldElems) * kFieldElems;
    chunks = cdiv(mesh.n, per);
    DevBuf part;
    part.alloc(sizeof(double2) * chunks * m);
    ProfScope prof(SB_PROF_OTHER, s);
    k_field<<<dim3(static_cast<unsigned>(tiles), static_cast<unsigned>(chunks)), kFieldPoints, 0, s>>>(
        mesh.elem.as<double>(), mesh.n, mesh.ld, pressure, velocity, ph.harmonic_factor * ph.wave_number,
        ph.pressure_factor, points, m, per, part.as<double2>());
    count_launch();
    SB_CUDA(cudaGetLastError());
    k_field_sum<<<static_cast<unsigned>(cdiv(m, 256)), 256, 0, s>>>(part.as<double2>(), m, static_cast<int>(chunks),
                                                                     out);
    count_launch();
    SB_CUDA(cudaGetLastError());
    SB_CUDA(cudaStreamSynchronize(s));
}

}  // namespace sb
