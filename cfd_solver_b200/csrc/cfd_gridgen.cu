// cfd_gridgen.cu -- the analytic grids of the two case profiles, generated on the GPU:
// coordinates, metrics (xi_x, xi_y, eta_x, eta_y, alpha, beta, gamma, J) and the boundary
// normals of INP.DAT (PSolver.cpp:517-547 reads them; the reference has no generator).
//
// O-grid: elliptic coordinates (mu, theta) around the cylinder x = c cosh(mu) cos(theta),
// y = c sinh(mu) sin(theta) with semi-axes 1 and 1/ar (log-polar r = exp(mu) for ar = 1),
// theta = 2 pi xi, mu = mu0 + L f(xi, eta), f = eta + s eta(1-eta) sin(2 pi xi).
// Cavity: x = xi + s xi(1-xi) sin(2 pi eta), y = eta + s eta(1-eta) sin(2 pi xi).
// The metrics come from the map's analytic derivatives: J = x_xi y_eta - x_eta y_xi,
// xi_x = y_eta / J, xi_y = -x_eta / J, eta_x = -y_xi / J, eta_y = x_xi / J,
// alpha = xi_x^2 + xi_y^2, gamma = eta_x^2 + eta_y^2, beta = -(xi_x eta_x + xi_y eta_y).
#include <cuda_runtime.h>

#include <cmath>
#include <string>
#include <vector>

#include "../../include/cfd_b200.h"

void cfd_internal_set_error(const char* msg);  // cfd_api.cu: read back by cfd_last_error()

namespace cfd {
namespace {
void set_last_error(const std::string& msg) { cfd_internal_set_error(msg.c_str()); }

struct GenArgs {
    int ogrid, n0, n1;
    int circle;       // O-grid with ar == 1: log-polar map
    double c, mu0, L;  // O-grid focal distance, inner mu, mu range
    double skew;
};

constexpr int GEN_THREADS = 256;

__global__ void __launch_bounds__(GEN_THREADS) k_grid_gen(GenArgs a, double* planes, double* normals) {
    const long long np = (long long)a.n0 * a.n1;
    const long long e = (long long)blockIdx.x * GEN_THREADS + threadIdx.x;
    if (e >= np) return;
    const int j = (int)(e / a.n0), i = (int)(e % a.n0);
    // the O-grid's seam column repeats column 0 exactly
    const int is = (a.ogrid && i == a.n0 - 1) ? 0 : i;
    const double two_pi = 2.0 * M_PI;
    const double xi = (double)is / (a.n0 - 1), eta = (double)j / (a.n1 - 1);
    const double s = a.skew;
    double x, y, x_xi, x_eta, y_xi, y_eta;
    if (a.ogrid) {
        const double th = two_pi * xi;
        const double sxi = sin(two_pi * xi), cxi = cos(two_pi * xi);
        const double f = eta + s * eta * (1.0 - eta) * sxi;
        const double f_xi = s * eta * (1.0 - eta) * two_pi * cxi;
        const double f_eta = 1.0 + s * (1.0 - 2.0 * eta) * sxi;
        const double mu = a.mu0 + a.L * f, mu_xi = a.L * f_xi, mu_eta = a.L * f_eta;
        const double ct = cos(th), st = sin(th);
        double x_mu, x_th, y_mu, y_th;
        if (!a.circle) {
            const double ch = cosh(mu), sh = sinh(mu);
            x = a.c * ch * ct;
            y = a.c * sh * st;
            x_mu = a.c * sh * ct;
            x_th = -a.c * ch * st;
            y_mu = a.c * ch * st;
            y_th = a.c * sh * ct;
        } else {
            const double r = exp(mu);
            x = r * ct;
            y = r * st;
            x_mu = r * ct;
            x_th = -r * st;
            y_mu = r * st;
            y_th = r * ct;
        }
        x_xi = x_mu * mu_xi + x_th * two_pi;
        y_xi = y_mu * mu_xi + y_th * two_pi;
        x_eta = x_mu * mu_eta;
        y_eta = y_mu * mu_eta;
    } else {
        const double se = sin(two_pi * eta), sx = sin(two_pi * xi);
        x = xi + s * xi * (1.0 - xi) * se;
        y = eta + s * eta * (1.0 - eta) * sx;
        x_xi = 1.0 + s * (1.0 - 2.0 * xi) * se;
        x_eta = s * xi * (1.0 - xi) * two_pi * cos(two_pi * eta);
        y_xi = s * eta * (1.0 - eta) * two_pi * cos(two_pi * xi);
        y_eta = 1.0 + s * (1.0 - 2.0 * eta) * sx;
    }
    const double jac = x_xi * y_eta - x_eta * y_xi;
    const double xix = y_eta / jac, xiy = -x_eta / jac, etx = -y_xi / jac, ety = x_xi / jac;
    const double alph = xix * xix + xiy * xiy, gam = etx * etx + ety * ety;
    const double beta = -(xix * etx + xiy * ety);
    const double v[10] = {x, y, xix, xiy, etx, ety, alph, beta, gam, jac};
#pragma unroll
    for (int q = 0; q < 10; q++) planes[(long long)q * np + e] = v[q];
    // boundary normals into the fluid: inner (j = 0) along +grad(eta), outer along -grad(eta)
    if (j == 0 || j == a.n1 - 1) {
        const double ge = sqrt(gam);
        const int off = j == 0 ? 0 : 2;
        const double sg = j == 0 ? 1.0 : -1.0;
        normals[(long long)off * a.n0 + i] = sg * etx / ge;
        normals[(long long)(off + 1) * a.n0 + i] = sg * ety / ge;
    }
}

}  // namespace
}  // namespace cfd

using namespace cfd;

namespace {
// Map parameters of `s`, or CFD_E_ARG (with the reason) for an invalid spec.
int gen_args(const cfd_grid_spec& s, GenArgs& a) {
    a = GenArgs{};
    a.n0 = s.n0;
    a.n1 = s.n1;
    a.skew = s.skew;
    if (s.n0 > 65536 || s.n1 > 65536) {
        set_last_error("grid generation: n0, n1 must be <= 65536");
        return CFD_E_ARG;
    }
    if (s.profile == CFD_PROFILE_OGRID) {
        if (s.n0 < 8 || s.n1 < 6 || !(s.ar >= 1.0) || !(s.r_outer > 1.0)) {
            set_last_error("grid generation: O-grid needs n0 >= 8, n1 >= 6, ar >= 1, r_outer > 1");
            return CFD_E_ARG;
        }
        a.ogrid = 1;
        if (s.ar > 1.0) {
            const double A = 1.0, B = 1.0 / s.ar;
            a.c = std::sqrt(A * A - B * B);
            a.mu0 = std::atanh(B / A);
            if (!(s.r_outer > a.c)) {
                set_last_error("grid generation: r_outer must exceed the focal distance");
                return CFD_E_ARG;
            }
            a.L = std::acosh(s.r_outer / a.c) - a.mu0;
        } else {
            a.circle = 1;
            a.mu0 = 0.0;
            a.L = std::log(s.r_outer);
        }
    } else if (s.profile == CFD_PROFILE_CAVITY) {
        if (s.n0 < 7 || s.n1 < 7) {
            set_last_error("grid generation: the cavity needs n0, n1 >= 7");
            return CFD_E_ARG;
        }
    } else {
        set_last_error("grid generation: unknown profile");
        return CFD_E_ARG;
    }
    return CFD_OK;
}
}  // namespace

// Checks `spec` and launches the generator on `stream`: 10 planes of n1 * n0 doubles into
// d_planes, 4 rows of n0 normals into d_normals (device memory). CFD_E_ARG for an invalid
// spec, before any device work. Also used by cfd_batch_admit_spec (cfd_api.cu).
int cfd_internal_grid_gen(const cfd_grid_spec* spec, double* d_planes, double* d_normals, cudaStream_t stream) {
    if (!spec) {
        set_last_error("grid generation: null spec");
        return CFD_E_ARG;
    }
    GenArgs a;
    if (int rc = gen_args(*spec, a)) return rc;
    const long long np = (long long)spec->n0 * spec->n1;
    const int blocks = (int)((np + GEN_THREADS - 1) / GEN_THREADS);
    k_grid_gen<<<blocks, GEN_THREADS, 0, stream>>>(a, d_planes, d_normals);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        set_last_error(std::string("grid generation: ") + cudaGetErrorString(e));
        return CFD_E_CUDA;
    }
    return CFD_OK;
}

extern "C" int cfd_grid_generate(const cfd_grid_spec* spec, double* planes, double* normals) {
    if (!spec || !planes || !normals) {
        set_last_error("cfd_grid_generate: null argument");
        return CFD_E_ARG;
    }
    const cfd_grid_spec& s = *spec;
    GenArgs a;
    if (int rc = gen_args(s, a)) return rc;  // an invalid spec touches no device
    const long long np = (long long)s.n0 * s.n1;
    const size_t nb = sizeof(double) * (size_t)(10 * np + 4LL * s.n0);
    double* d = nullptr;
    if (cudaMalloc((void**)&d, nb) != cudaSuccess) {
        set_last_error("cfd_grid_generate: no device memory");
        return CFD_E_OOM;
    }
    const int rc = cfd_internal_grid_gen(spec, d, d + 10 * np, 0);
    if (rc != CFD_OK) {
        cudaFree(d);
        return rc;
    }
    cudaError_t e = cudaMemcpy(planes, d, sizeof(double) * 10 * np, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(normals, d + 10 * np, sizeof(double) * 4 * s.n0, cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (e != cudaSuccess) {
        set_last_error(std::string("cfd_grid_generate: ") + cudaGetErrorString(e));
        return CFD_E_CUDA;
    }
    return CFD_OK;
}
