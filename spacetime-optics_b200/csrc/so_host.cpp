// so_host.cpp -- host-side utilities of the C ABI that need no renderer: metric functions at a point,
// the analytic critical curve, the star-map file reader, the far-field approach check and the torus
// plasma's Fourier modes.
#include <algorithm>
#include <cmath>
#include <cstdio>

#include "so_kerr.cuh"

using namespace so;

extern "C" {

void so_kerr_point_at(double a, double r, double th, so_kerr_point* kp) {
    if (kp) kerr_point(a, r, th, kp);
}

int so_critical_curve_point(double a, double theta_o, double rp, double* alpha, double* beta_plus) {
    if (!alpha || !beta_plus) return 0;
    return critical_curve_point(a, theta_o, rp, alpha, beta_plus) ? 1 : 0;
}

int so_sky_file(const char* path, int* w, int* h, float* scale, uint16_t* data) {
    if (!path || !w || !h || !scale) return SO_ERR_ARG;
    FILE* f = std::fopen(path, "rb");
    if (!f) return SO_ERR_CONFIG;
    uint32_t hdr[3];
    float sc = 0.f;
    if (std::fread(hdr, 4, 3, f) != 3 || hdr[0] != 0x4b534842u || std::fread(&sc, 4, 1, f) != 1 || hdr[1] == 0 ||
        hdr[2] == 0 || (uint64_t)hdr[1] * hdr[2] > (1ull << 28)) {
        std::fclose(f);
        return SO_ERR_CONFIG;
    }
    *w = (int)hdr[1];
    *h = (int)hdr[2];
    *scale = sc;
    int rc = SO_OK;
    if (data) {
        const size_t n = (size_t)hdr[1] * hdr[2] * 2;
        if (std::fread(data, 2, n, f) != n) rc = SO_ERR_CONFIG;
    }
    std::fclose(f);
    return rc;
}

int so_approach_state(const so_scene* S, const so_frame* f, double x, double yv, double r1, double tol, int method,
                      double* state, int* attempts) {
    if (!S || !f || !state || !(r1 > 0.0) || !(tol > 0.0) || (method != 0 && method != 1)) return SO_ERR_ARG;
    RayC c;
    double y[6];
    camera_photon(S->a, f->kp, f->ph, f->t, view_dir(*f, x, yv), f->beta, c, y);
    int att = 0;
    if (method == 0) {
        if (!far_applies(c, y, r1)) return SO_ERR_ARG;
        double psi = 0.0;
        int nc = 0;
        att = far_approach(c, y, r1, tol, 100000, &psi, &nc, false);
        if (att < 0) return SO_ERR_STATE;
    } else {
        // Mino-time DP5(4) with the reference's controller; a step that would pass r1 is shortened
        // (secant in r) until the ray stops within 1e-12 r1 above r1
        if (!(y[0] > r1) || !(y[1] < 0.0)) return SO_ERR_ARG;
        double k1[6], yn[6], k7[6];
        rhs(c, y, k1);
        double h = initial_step(y);
        while (y[0] - r1 > 1e-12 * r1) {
            if (++att > 10000000) return SO_ERR_STATE;
            const double hc = h;
            const double err = dp54(c, y, k1, hc, tol, yn, k7);
            if (!(err <= 1.0)) {
                h = reject_step(hc, err);
                continue;
            }
            if (yn[0] < r1) {
                h = hc * (y[0] - r1) / (y[0] - yn[0]) * (1.0 - 1e-13);
                continue;
            }
            for (int i = 0; i < 6; ++i) {
                y[i] = yn[i];
                k1[i] = k7[i];
            }
            project_radial(c, y, k1);
            if (y[1] >= 0.0) return SO_ERR_ARG;  // radial turning point above r1
            h = accept_step(hc, err);
        }
    }
    for (int i = 0; i < 6; ++i) state[i] = y[i];
    if (attempts) *attempts = att;
    return SO_OK;
}

// Torus turbulence modes (so_tracer.h): directions uniform on the sphere, |k| log-uniform in
// [k_min, k_max], phases uniform, amplitude^2 proportional to |k|^(3 + spectral_index) -- the
// variance per logarithmic k interval of a 3-D power spectrum P(k) ~ k^spectral_index -- scaled so
// that sum amp^2 / 2 = turb_rms^2.  Random numbers: the pcg hash of device_util.cuh:15-19 chained
// from turb_seed.
int so_plasma_modes(const so_plasma* p, so_mode* modes) {
    if (!p || !modes || p->n_modes < 0 || p->n_modes > SO_MAX_MODES || !(p->k_min > 0) || !(p->k_max >= p->k_min))
        return SO_ERR_ARG;
    auto pcg_h = [](uint32_t v) {
        uint32_t s = v * 747796405u + 2891336453u;
        uint32_t w = ((s >> ((s >> 28u) + 4u)) ^ s) * 277803737u;
        return (w >> 22u) ^ w;
    };
    uint32_t st = pcg_h(p->turb_seed ^ 0x7f4a7c15u);
    auto uni = [&]() {
        st = pcg_h(st);
        return (double)(st >> 8) * (1.0 / 16777216.0);
    };
    double wsum = 0.0;
    for (int m = 0; m < p->n_modes; ++m) {
        double cz = 2.0 * uni() - 1.0, az = 2.0 * PI * uni();
        double sz = std::sqrt(std::max(0.0, 1.0 - cz * cz));
        double k = p->k_min * std::pow(p->k_max / p->k_min, uni());
        modes[m].kx = k * sz * std::cos(az);
        modes[m].ky = k * sz * std::sin(az);
        modes[m].kz = k * cz;
        modes[m].phase = 2.0 * PI * uni();
        double w = std::pow(k, 3.0 + p->spectral_index);
        modes[m].amp = w;
        wsum += w;
    }
    for (int m = 0; m < p->n_modes; ++m) modes[m].amp = p->turb_rms * std::sqrt(2.0 * modes[m].amp / wsum);
    return SO_OK;
}

}  // extern "C"
