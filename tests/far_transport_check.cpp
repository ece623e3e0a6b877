// Host check of the inverse-radius transport (far_approach in so_kerr.cuh) against the Mino-time
// DP5(4) at tolerance 1e-13, on the synchrotron camera (a = 0.94, i = 163 deg, r = 1e7 M):
//   outwards: rays past their periapsis, from r ~ 60 M to r = 1000 M (the escape leg);
// prints one line per ray: attempts of both integrators and the state differences.  Built and run
// by tests/test_far_transport.py (test infrastructure, no device).
#include <cmath>
#include <cstdio>

#include "so_kerr.cuh"
using namespace so;

// Mino-time DP5(4) from y until r reaches r1 moving in its current radial direction (the last step
// shortened by secant in r to stop within 1e-12 r1 of r1).
static int mino_to(const RayC& c, double* y, double r1, double tol) {
    double k1[6], yn[6], k7[6];
    rhs(c, y, k1);
    double h = initial_step(y);
    int att = 0;
    const bool out = r1 > y[0];
    while (std::fabs(y[0] - r1) > 1e-12 * r1) {
        if (++att > 4000000) return -1;
        const double hc = h;
        const double err = dp54(c, y, k1, hc, tol, yn, k7);
        if (!(err <= 1.0)) {
            h = reject_step(hc, err);
            continue;
        }
        const bool past = out ? yn[0] > r1 : yn[0] < r1;
        if (past) {
            h = hc * (r1 - y[0]) / (yn[0] - y[0]) * (1.0 - 1e-13);
            continue;
        }
        for (int i = 0; i < 6; ++i) {
            y[i] = yn[i];
            k1[i] = k7[i];
        }
        project_radial(c, y, k1);
        h = accept_step(hc, err);
    }
    return att;
}

int main() {
    const double a = 0.94, rc = 1e7, th = 163.0 * PI / 180.0;
    so_kerr_point kp;
    kerr_point(a, rc, th, &kp);
    const so_vec3 beta = {0.0, 0.0, 0.0};
    for (int k = 0; k < 12; ++k) {
        const double al = 8.0 + 0.9 * k, be = -6.0 + k;  // outside the shadow: escaping rays
        const double nx = -1.0, ny = -be / rc, nz = al / rc, il = 1.0 / std::sqrt(nx * nx + ny * ny + nz * nz);
        const so_vec3 d = {nx * il, ny * il, nz * il};
        RayC c;
        double y[6], k1[6], yn[6], k7[6];
        camera_photon(a, kp, 0.3, 0.0, d, beta, c, y);
        rhs(c, y, k1);
        double h = initial_step(y);
        for (int it = 0; it < 4000000 && !(y[1] > 0.0 && y[0] > 60.0) && y[0] > 2.0; ++it) {
            const double hc = h, err = dp54(c, y, k1, hc, 1e-13, yn, k7);
            if (!(err <= 1.0)) {
                h = reject_step(hc, err);
                continue;
            }
            for (int i = 0; i < 6; ++i) {
                y[i] = yn[i];
                k1[i] = k7[i];
            }
            project_radial(c, y, k1);
            h = accept_step(hc, err);
        }
        if (!(y[1] > 0.0 && y[0] > 60.0)) {
            std::printf("skip\n");
            continue;
        }
        double ym[6], yf[6];
        for (int i = 0; i < 6; ++i) ym[i] = yf[i] = y[i];
        const int nm = mino_to(c, ym, 1000.0, 1e-13);
        double psi = 0.0;
        int nc = 0;
        const int applies = far_applies(c, yf, ym[0]) ? 1 : 0;
        const int nf = applies ? far_approach(c, yf, ym[0], 1e-9, 256, &psi, &nc, false) : -1;
        std::printf("%d %d %d %.3e %.3e %.3e %.3e %.3e %.3e\n", applies, nm, nf, std::fabs(yf[0] - ym[0]),
                    std::fabs(yf[1] - ym[1]) / std::fabs(ym[1]), std::fabs(yf[2] - ym[2]), std::fabs(yf[3] - ym[3]),
                    std::fabs(yf[4] - ym[4]), std::fabs(yf[5] - ym[5]));
    }
    return 0;
}
