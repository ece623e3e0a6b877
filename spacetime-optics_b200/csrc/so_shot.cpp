// so_shot.cpp -- shot .ini -> so_scene / so_frame (host).  Restates the reference's host builders so
// that bhrt shot files drop in:
//   INI reader            common/config.cpp:45-134 (sections, '#' comments, '\' continuation,
//                         top-level include, section.key addressing) and --set (main.cpp:389-399)
//   build_scene           blackholes/src/scene_build.cpp:83-213 (defaults, spin clamp, NT flux
//                         table :26-59 / :116-141, ln K2 table :159-170, blackbody table colour.cpp)
//   build_shot / Track    blackholes/src/shot.cpp:29-114 (monotone cubic tracks)
//   make_frame            blackholes/src/shot.cpp:116-146
//   find_critical_point   blackholes/src/shot.cpp:148-164 (host FP64 bisection on vacuum_fate)
// plus the torus-plasma keys of the [so] section, which the reference does not have.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <vector>

#include "so_kerr.cuh"

namespace so {
namespace {

std::string trim(const std::string& s) {
    size_t a = s.find_first_not_of(" \t\r\n");
    if (a == std::string::npos) return "";
    size_t b = s.find_last_not_of(" \t\r\n");
    return s.substr(a, b - a + 1);
}

struct Config {
    std::map<std::string, std::string> kv;
    std::string dir;

    bool load(const std::string& path, std::string* err) {
        std::ifstream in(path);
        if (!in) {
            *err = "cannot open " + path;
            return false;
        }
        size_t slash = path.find_last_of('/');
        dir = slash == std::string::npos ? "." : path.substr(0, slash);
        std::string raw, section;
        int lineno = 0;
        while (std::getline(in, raw)) {
            ++lineno;
            std::string line = raw;
            size_t c = line.find('#');
            if (c != std::string::npos) line = line.substr(0, c);
            line = trim(line);
            while (!line.empty() && line.back() == '\\' && std::getline(in, raw)) {
                ++lineno;
                line.pop_back();
                size_t c2 = raw.find('#');
                line += " " + trim(c2 == std::string::npos ? raw : raw.substr(0, c2));
                line = trim(line);
            }
            if (line.empty()) continue;
            if (line.front() == '[') {
                if (line.back() != ']') {
                    *err = path + ":" + std::to_string(lineno) + ": bad section header";
                    return false;
                }
                section = trim(line.substr(1, line.size() - 2));
                continue;
            }
            size_t eq = line.find('=');
            if (eq == std::string::npos) {
                *err = path + ":" + std::to_string(lineno) + ": expected key = value";
                return false;
            }
            std::string key = trim(line.substr(0, eq)), val = trim(line.substr(eq + 1));
            if (section.empty() && key == "include") {
                std::string d = dir;
                if (val.empty() || !load(val[0] == '/' ? val : d + "/" + val, err)) {
                    if (err->empty()) *err = path + ": empty include";
                    return false;
                }
                dir = d;
                continue;
            }
            kv[section.empty() ? key : section + "." + key] = val;
        }
        return true;
    }
    bool has(const std::string& k) const { return kv.count(k) != 0; }
    std::string str(const std::string& k, const std::string& def = "") const {
        auto it = kv.find(k);
        return it == kv.end() ? def : it->second;
    }
    double num(const std::string& k, double def) const {
        auto it = kv.find(k);
        if (it == kv.end() || it->second.empty()) return def;
        char* end = nullptr;
        double v = std::strtod(it->second.c_str(), &end);
        return end == it->second.c_str() ? def : v;
    }
    int integer(const std::string& k, int def) const { return (int)num(k, def); }
    bool flag(const std::string& k, bool def) const {
        auto it = kv.find(k);
        if (it == kv.end()) return def;
        const std::string& v = it->second;
        if (v == "1" || v == "true" || v == "yes" || v == "on") return true;
        if (v == "0" || v == "false" || v == "no" || v == "off") return false;
        return def;
    }
};

// Circular equatorial prograde orbits, M = 1 (scene_build.cpp:12-20).
double orb_E(double a, double r) {
    double sr = std::sqrt(r);
    return (r * sr - 2.0 * sr + a) / (std::pow(r, 0.75) * std::sqrt(r * sr - 3.0 * sr + 2.0 * a));
}
double orb_L(double a, double r) {
    double sr = std::sqrt(r);
    return (r * r - 2.0 * a * sr + a * a) / (std::pow(r, 0.75) * std::sqrt(r * sr - 3.0 * sr + 2.0 * a));
}
double orb_Om(double a, double r) { return 1.0 / (r * std::sqrt(r) + a); }

double isco_radius(double a) {  // kerr.hpp:96-100
    double z1 = 1.0 + std::cbrt(1.0 - a * a) * (std::cbrt(1.0 + a) + std::cbrt(1.0 - a));
    double z2 = std::sqrt(3.0 * a * a + z1 * z1);
    return 3.0 + z2 - std::sqrt((3.0 - z1) * (3.0 + z1 + 2.0 * z2));
}

// Page-Thorne flux for Mdot = 1 (scene_build.cpp:26-58): trapezoid integral of (E - Om L) dL/dr on a
// 200000-point log grid from the ISCO, linear interpolation at the requested radii.
std::vector<double> nt_flux(double a, const std::vector<double>& r) {
    double risco = isco_radius(a);
    std::vector<double> F(r.size(), 0.0);
    const int N = 200000;
    double lr0 = std::log(risco), lr1 = std::log(r.back());
    std::vector<double> rg(N), I(N, 0.0);
    for (int i = 0; i < N; ++i) rg[i] = std::exp(lr0 + (lr1 - lr0) * i / (N - 1));
    auto integrand = [&](double x) {
        double h = 1e-6 * x;
        double Lr = (orb_L(a, x + h) - orb_L(a, x - h)) / (2 * h);
        return (orb_E(a, x) - orb_Om(a, x) * orb_L(a, x)) * Lr;
    };
    double prev = integrand(rg[0] * (1 + 1e-9));
    for (int i = 1; i < N; ++i) {
        double cur = integrand(rg[i]);
        I[i] = I[i - 1] + 0.5 * (prev + cur) * (rg[i] - rg[i - 1]);
        prev = cur;
    }
    for (size_t j = 0; j < r.size(); ++j) {
        double x = r[j];
        if (x <= risco) continue;
        double fi = (std::log(x) - lr0) / (lr1 - lr0) * (N - 1);
        int i = std::min(std::max((int)fi, 0), N - 2);
        double Ix = I[i] + (I[i + 1] - I[i]) * (fi - i);
        double Omr = -1.5 * std::sqrt(x) / std::pow(x * std::sqrt(x) + a, 2);
        double EmOL = orb_E(a, x) - orb_Om(a, x) * orb_L(a, x);
        F[j] = -Omr / (4.0 * PI * x * EmOL * EmOL) * Ix;
    }
    return F;
}

// CIE 1931 2-degree standard observer, 380..780 nm in 10 nm steps (the published CIE table).
const double CIE_X[41] = {0.001368, 0.004243, 0.014310, 0.043510, 0.134380, 0.283900, 0.348280, 0.336200,
                          0.290800, 0.195360, 0.095640, 0.032010, 0.004900, 0.009300, 0.063270, 0.165500,
                          0.290400, 0.433450, 0.594500, 0.762100, 0.916300, 1.026300, 1.062200, 1.002600,
                          0.854450, 0.642400, 0.447900, 0.283500, 0.164900, 0.087400, 0.046770, 0.022700,
                          0.011359, 0.005790, 0.002899, 0.001440, 0.000690, 0.000332, 0.000166, 0.000083,
                          0.000042};
const double CIE_Y[41] = {0.000039, 0.000120, 0.000396, 0.001210, 0.004000, 0.011600, 0.023000, 0.038000,
                          0.060000, 0.090980, 0.139020, 0.208020, 0.323000, 0.503000, 0.710000, 0.862000,
                          0.954000, 0.994950, 0.995000, 0.952000, 0.870000, 0.757000, 0.631000, 0.503000,
                          0.381000, 0.265000, 0.175000, 0.107000, 0.061000, 0.032000, 0.017000, 0.008210,
                          0.004102, 0.002091, 0.001047, 0.000520, 0.000249, 0.000120, 0.000060, 0.000030,
                          0.000015};
const double CIE_Z[41] = {0.006450, 0.020050, 0.067850, 0.207400, 0.645600, 1.385600, 1.747060, 1.772110,
                          1.669200, 1.287640, 0.812950, 0.465180, 0.272000, 0.158200, 0.078250, 0.042160,
                          0.020300, 0.008750, 0.003900, 0.002100, 0.001650, 0.001100, 0.000800, 0.000340,
                          0.000190, 0.000050, 0.000020, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
double cmf(const double* t, double lam) {  // linear interpolation of the 10 nm table
    double x = (lam - 380.0) / 10.0;
    if (x <= 0) return t[0];
    if (x >= 40) return t[40];
    int i = (int)x;
    double f = x - i;
    return t[i] * (1 - f) + t[i + 1] * f;
}
// Spectral radiance of a blackbody per nm (W m^-2 sr^-1 nm^-1), SI constants.
double planck_nm(double lambda_nm, double T) {
    const double h = 6.62607015e-34, c = 299792458.0, k = 1.380649e-23;
    double l = lambda_nm * 1e-9;
    return 2.0 * h * c * c / (l * l * l * l * l) / std::expm1(h * c / (l * k * T)) * 1e-9;
}
// XYZ of B(T) on a ln T grid from 300 K to 3e7 K, 2048 entries (colour.cpp:49-63 layout).
std::vector<float> blackbody_table(float* l0, float* dl) {
    const int N = 2048;
    double a = std::log(300.0), b = std::log(3e7), d = (b - a) / (N - 1);
    std::vector<float> t(3 * N);
    for (int i = 0; i < N; ++i) {
        double T = std::exp(a + i * d), xyz[3] = {0, 0, 0};
        for (double lam = 380.5; lam < 780.0; lam += 1.0) {
            double bb = planck_nm(lam, T);
            xyz[0] += bb * cmf(CIE_X, lam);
            xyz[1] += bb * cmf(CIE_Y, lam);
            xyz[2] += bb * cmf(CIE_Z, lam);
        }
        for (int c = 0; c < 3; ++c) t[3 * i + c] = (float)xyz[c];
    }
    *l0 = (float)a;
    *dl = (float)d;
    return t;
}

// Animated parameter track (shot.cpp:29-71): "time:value, ..." with Fritsch-Carlson monotone cubic
// Hermite interpolation, zero end tangents, optionally in log space.
struct Track {
    std::vector<double> t, v;
    bool log = false;
    double value(double time) const {
        size_t n = t.size();
        double out;
        if (n == 1 || time <= t[0]) out = v[0];
        else if (time >= t[n - 1]) out = v[n - 1];
        else {
            size_t i = 0;
            while (i + 2 < n && time > t[i + 1]) ++i;
            auto sec = [&](size_t k) { return (v[k + 1] - v[k]) / (t[k + 1] - t[k]); };
            auto tan = [&](size_t k) {
                if (k == 0 || k == n - 1) return 0.0;
                double a = sec(k - 1), b = sec(k);
                if (a * b <= 0) return 0.0;
                double h0 = t[k] - t[k - 1], h1 = t[k + 1] - t[k];
                return 3.0 * (h0 + h1) / ((2.0 * h1 + h0) / a + (h1 + 2.0 * h0) / b);
            };
            double h = t[i + 1] - t[i], s = (time - t[i]) / h;
            double h00 = (1 + 2 * s) * (1 - s) * (1 - s), h10 = s * (1 - s) * (1 - s), h01 = s * s * (3 - 2 * s),
                   h11 = s * s * (s - 1);
            out = h00 * v[i] + h10 * h * tan(i) + h01 * v[i + 1] + h11 * h * tan(i + 1);
        }
        return log ? std::exp(out) : out;
    }
};

bool parse_track(const std::string& s, bool log, Track* tr) {
    std::stringstream ss(s);
    std::string item;
    while (std::getline(ss, item, ',')) {
        item = trim(item);
        if (item.empty()) continue;
        size_t c = item.find(':');
        if (c == std::string::npos) return false;
        double t = std::strtod(item.substr(0, c).c_str(), nullptr), v = std::strtod(item.substr(c + 1).c_str(), nullptr);
        tr->t.push_back(t);
        tr->v.push_back(log ? std::log(v) : v);
    }
    tr->log = log;
    return !tr->t.empty();
}

double param(const Config& c, const std::string& key, double def, double time, bool log) {
    std::string tk = "track." + key;
    if (c.has(tk)) {
        Track tr;
        if (parse_track(c.str(tk), log, &tr)) return tr.value(time);
    }
    return c.num(key, def);
}

so_vec3 v3(double x, double y, double z) {
    so_vec3 v = {x, y, z};
    return v;
}
so_vec3 add(so_vec3 a, so_vec3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
so_vec3 mul(so_vec3 a, double s) { return v3(a.x * s, a.y * s, a.z * s); }
double dotp(so_vec3 a, so_vec3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
so_vec3 crossp(so_vec3 a, so_vec3 b) {
    return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
so_vec3 rotate(so_vec3 v, so_vec3 axis, double ang) {  // Rodrigues (shot.cpp:43-46)
    double cs = std::cos(ang), sn = std::sin(ang);
    return add(add(mul(v, cs), mul(crossp(axis, v), sn)), mul(axis, dotp(axis, v) * (1 - cs)));
}

struct ShotFrame {
    double t = 0, r = 0, incl = 0, phi = 0, roll = 0, yaw = 0, pitch = 0, fov = 0;
    bool fov_in_m = false;
    double zoom = 1, target = 0, off_x = 0, off_y = 0, time_m = 0;
};

}  // namespace

// Scene scalars of the vacuum geodesics for spin a (the scene builder's clamp, horizon, ISCO and
// stopping radius with the same horizon margin); the tables and the emitters' parameters stay.
void scene_set_spin(so_scene* S, double a) {
    const double margin = S->r_stop - S->rh;
    if (a <= 0.0) a = 1e-6;
    if (a > 0.9999) a = 0.9999;
    S->a = a;
    S->rh = horizon_radius(a);
    S->r_isco = isco_radius(a);
    S->r_stop = S->rh + margin;
}

void set_global_error(const std::string& msg);  // so_renderer.cpp: so_last_error(NULL)
}  // namespace so

using namespace so;

struct so_shot {
    Config cfg;
    so_scene S;
    so_scene_info info;
    std::vector<float> disk_lnT, k2_ln, bb_xyz;
    std::string name, type, motion;
    double duration = 5, fps = 30, target_x = 0, target_y = 0;
    std::vector<ShotFrame> frames;
};

namespace {

bool build_scene(so_shot* sh, std::string* err) {
    const Config& c = sh->cfg;
    so_scene* S = &sh->S;
    std::memset(S, 0, sizeof(so_scene));
    double a = c.num("bh.spin", 0.94);
    if (a <= 0.0) a = 1e-6;  // the formulas use 1/a (scene_build.cpp:86)
    if (a > 0.9999) a = 0.9999;
    S->a = a;
    S->rh = horizon_radius(a);
    S->r_isco = isco_radius(a);
    S->tol = c.num("render.tolerance", 1e-9);
    S->max_steps = c.integer("render.max_steps", 20000);
    S->r_escape = c.num("render.r_escape", 2e4);
    S->r_stop = S->rh + c.num("render.horizon_margin", 0.01);
    S->step_frac = c.num("render.step_fraction", 0.04);
    S->mode = c.str("render.mode", "visible") == "radio" ? SO_MODE_RADIO : SO_MODE_VISIBLE;
    S->seed = (uint32_t)c.integer("render.seed", 1) * 2654435761u;

    so_scene_info& info = sh->info;
    std::memset(&info, 0, sizeof info);
    info.mass_msun = c.num("bh.mass_msun", 6.5e9);
    double dist_pc = c.has("bh.distance_mpc") ? c.num("bh.distance_mpc", 16.8) * 1e6 : c.num("bh.distance_pc", 16.8e6);
    const double PC = 3.0856775814913673e18, G = 6.67430e-8, MSUN = 1.98847e33, CC = 2.99792458e10;
    info.distance_cm = dist_pc * PC;
    info.rg_cm = G * info.mass_msun * MSUN / (CC * CC);
    info.tg_s = info.rg_cm / CC;
    info.uas_per_m = info.rg_cm / info.distance_cm * (180.0 / PI * 3600.0e6);

    S->disk_on = c.flag("disk.enabled", S->mode == SO_MODE_VISIBLE) ? 1 : 0;
    S->disk_rin = std::max(c.num("disk.r_in", 0.0), S->r_isco);
    S->disk_rout = c.num("disk.r_out", 40.0);
    S->disk_turb_amp = (float)c.num("disk.turbulence", 0.45);
    S->disk_turb_scale = (float)c.num("disk.turbulence_scale", 0.35);
    S->disk_tcorr = (float)c.num("disk.correlation_orbits", 0.6);
    S->disk_ld = c.flag("disk.limb_darkening", true) ? 1.f : 0.f;
    S->disk_fcol = (float)c.num("disk.color_correction", 1.0);
    {
        const int N = 1024;
        double l0 = std::log(S->r_isco * 1.0001), l1 = std::log(S->disk_rout * 1.05);
        std::vector<double> r(N);
        for (int i = 0; i < N; ++i) r[i] = std::exp(l0 + (l1 - l0) * i / (N - 1));
        std::vector<double> F = nt_flux(a, r);
        double eta = 1.0 - orb_E(a, S->r_isco);
        double LEdd = 1.26e38 * info.mass_msun;
        double fedd = c.num("disk.eddington_ratio", 0.1);
        double Mdot = fedd * LEdd / (eta * CC * CC);
        const double sigma = 5.670374419e-5;
        double fmx = *std::max_element(F.begin(), F.end());
        double Tmax_phys = std::pow(fmx * Mdot * CC * CC / (info.rg_cm * info.rg_cm) / sigma, 0.25);
        double Tmax = c.num("disk.t_max", Tmax_phys);
        info.disk_tmax = Tmax;
        info.disk_mdot_edd = fedd * std::pow(Tmax / Tmax_phys, 4.0);
        sh->disk_lnT.resize(N);
        for (int i = 0; i < N; ++i) {
            double Ti = Tmax * std::pow(std::max(F[i], 1e-300) / fmx, 0.25);
            sh->disk_lnT[i] = (float)std::log(std::max(Ti, 1.0));
        }
        S->disk_n = N;
        S->disk_lr0 = l0;
        S->disk_dlr = (l1 - l0) / (N - 1);
    }

    S->flow_on = c.flag("flow.enabled", S->mode == SO_MODE_RADIO) ? 1 : 0;
    S->n0 = c.num("flow.n0", 1e5);
    S->n_index = c.num("flow.n_index", 1.1);
    S->theta0 = c.num("flow.theta0", 25.0);
    S->theta_index = c.num("flow.theta_index", 0.84);
    S->h_r = c.num("flow.h_over_r", 0.4);
    S->beta_p = c.num("flow.beta", 10.0);
    S->r_flow_max = c.num("flow.r_max", 60.0);
    S->nu_obs = c.num("flow.nu_ghz", 230.0) * 1e9;
    S->rg_cm = info.rg_cm;
    S->flow_kep = c.num("flow.keplerian_fraction", 0.9);
    S->flow_turb_amp = (float)c.num("flow.turbulence", 0.7);
    S->flow_turb_scale = (float)c.num("flow.turbulence_scale", 0.45);
    S->flow_tcorr = (float)c.num("flow.correlation_orbits", 0.5);
    info.radio_flux_target_jy = c.num("flow.flux_jy", 0.0);
    {
        const int N = 512;
        double l0 = std::log(0.02), l1 = std::log(1e4);
        sh->k2_ln.resize(N);
        for (int i = 0; i < N; ++i) {
            double th = std::exp(l0 + (l1 - l0) * i / (N - 1));
            sh->k2_ln[i] = (float)std::log(std::cyl_bessel_k(2.0, 1.0 / th));
        }
        S->k2_n = N;
        S->k2_l0 = (float)l0;
        S->k2_dl = (float)((l1 - l0) / (N - 1));
    }
    // The celestial sphere needs the star-map texture, which this library does not carry.
    S->sky_on = c.flag("sky.enabled", S->mode == SO_MODE_VISIBLE) ? 1 : 0;
    S->sky_scale = (float)c.num("sky.brightness", 1.0);
    {
        double l = c.num("sky.l_deg", 0.0) * PI / 180, b = c.num("sky.b_deg", 0.0) * PI / 180;
        double incl = c.num("camera.incl", 80.0) * PI / 180, ph = c.num("camera.phi", 0.0) * PI / 180;
        double roll = c.num("sky.roll_deg", 0.0) * PI / 180;
        so_vec3 behind = v3(-(std::sin(incl) * std::cos(ph)), -(std::sin(incl) * std::sin(ph)), -std::cos(incl));
        so_vec3 z = v3(0, 0, 1);
        so_vec3 upv = add(z, mul(behind, -dotp(z, behind)));
        so_vec3 up = mul(upv, 1.0 / std::sqrt(dotp(upv, upv)));
        if (!(std::sqrt(dotp(up, up)) > 0.5)) up = v3(1, 0, 0);
        so_vec3 side = crossp(up, behind);
        so_vec3 gt = v3(std::cos(b) * std::cos(l), std::cos(b) * std::sin(l), std::sin(b));
        so_vec3 gnv = add(z, mul(gt, -dotp(z, gt)));
        so_vec3 gn = mul(gnv, 1.0 / std::sqrt(dotp(gnv, gnv)));
        so_vec3 gs = crossp(gn, gt);
        so_vec3 gu = add(mul(gn, std::cos(roll)), mul(gs, std::sin(roll)));
        so_vec3 gv = crossp(gu, gt);
        auto comp = [](so_vec3 v, int i) { return i == 0 ? v.x : i == 1 ? v.y : v.z; };
        so_vec3* rows[3] = {&S->sky_rot.r0, &S->sky_rot.r1, &S->sky_rot.r2};
        for (int i = 0; i < 3; ++i)
            *rows[i] = v3(comp(gt, i) * behind.x + comp(gu, i) * up.x + comp(gv, i) * side.x,
                          comp(gt, i) * behind.y + comp(gu, i) * up.y + comp(gv, i) * side.y,
                          comp(gt, i) * behind.z + comp(gu, i) * up.z + comp(gv, i) * side.z);
    }
    float bl0, bdl;
    sh->bb_xyz = blackbody_table(&bl0, &bdl);
    S->bb_n = 2048;
    S->bb_l0 = bl0;
    S->bb_dl = bdl;
    S->disk_lnT = sh->disk_lnT.data();
    S->k2_lntab = sh->k2_ln.data();
    S->bb_xyz = sh->bb_xyz.data();
    (void)err;
    return true;
}

void build_frames(so_shot* sh) {
    const Config& c = sh->cfg;
    sh->name = c.str("shot.name", "shot");
    sh->type = c.str("shot.type", "render");
    sh->duration = c.num("shot.duration", 5);
    sh->fps = c.num("shot.fps", 30);
    sh->motion = c.str("camera.motion", "static");
    int n = std::max(1, (int)std::lround(sh->duration * sh->fps));
    if (c.has("shot.frames")) n = c.integer("shot.frames", n);
    const double D2R = PI / 180;
    sh->frames.clear();
    for (int i = 0; i < n; ++i) {
        ShotFrame f;
        f.t = i / sh->fps;
        double t = f.t;
        f.r = param(c, "camera.r", 1e6, t, true);
        f.incl = param(c, "camera.incl", 80, t, false) * D2R;
        f.phi = param(c, "camera.phi", 0, t, false) * D2R;
        f.roll = param(c, "camera.roll", 0, t, false) * D2R;
        f.yaw = param(c, "camera.yaw", 0, t, false) * D2R;
        f.pitch = param(c, "camera.pitch", 0, t, false) * D2R;
        f.fov_in_m = c.has("camera.fov_m") || c.has("track.camera.fov_m");
        f.fov = f.fov_in_m ? param(c, "camera.fov_m", 30, t, true) : param(c, "camera.fov_deg", 40, t, true) * D2R;
        f.zoom = param(c, "camera.zoom", 1, t, true);
        f.target = param(c, "camera.target", 0, t, false);
        f.off_x = param(c, "camera.offset_x_m", 0, t, false);
        f.off_y = param(c, "camera.offset_y_m", 0, t, false);
        f.time_m = param(c, "time.t_m", 0, t, false);
        sh->frames.push_back(f);
    }
}

so_frame make_frame(const so_shot* sh, const ShotFrame& f, double a, int W, uint32_t seed) {
    so_frame F;
    std::memset(&F, 0, sizeof F);
    F.r = f.r;
    F.th = f.incl;
    F.ph = f.phi;
    F.t = f.time_m;
    kerr_point(a, f.r, f.incl, &F.kp);
    // Looking at the hole: forward = -e_r, up = -e_theta, right = e_phi (shot.cpp:123)
    so_vec3 Fw = v3(-1, 0, 0), Up = v3(0, -1, 0), Rt = v3(0, 0, 1);
    if (f.yaw != 0) {
        Fw = rotate(Fw, Up, -f.yaw);
        Rt = rotate(Rt, Up, -f.yaw);
    }
    if (f.pitch != 0) {
        Fw = rotate(Fw, Rt, f.pitch);
        Up = rotate(Up, Rt, f.pitch);
    }
    if (f.roll != 0) {
        Rt = rotate(Rt, Fw, f.roll);
        Up = rotate(Up, Fw, f.roll);
    }
    F.F = Fw;
    F.R = Rt;
    F.U = Up;
    double width = f.fov_in_m ? f.fov / f.r : 2.0 * std::tan(0.5 * f.fov);
    F.pix = width / f.zoom / W;
    if (f.fov_in_m) {
        F.cx = (f.off_x + f.target * sh->target_x) / f.r;
        F.cy = (f.off_y + f.target * sh->target_y) / f.r;
    }
    if (sh->motion == "orbit") {
        double Om = 1.0 / (std::pow(f.r, 1.5) + a);
        double v = (Om - F.kp.omega) * F.kp.e_psi / F.kp.e_nu;
        F.beta = v3(0, 0, std::max(-0.98, std::min(0.98, v)));
    }
    F.seed = seed;
    return F;
}

double find_critical(const so_shot* sh, const ShotFrame& f, double a, double psi) {
    so_frame F = make_frame(sh, f, a, 1, 0);
    auto fate = [&](double rho) {
        double x = rho * std::cos(psi) / f.r, y = rho * std::sin(psi) / f.r;
        so_frame G = F;
        G.cx = 0;
        G.cy = 0;
        return vacuum_fate(a, G, view_dir(G, x, y), 1e-12, 200.0, 2000000);
    };
    double lo = 0.5, hi = 15.0;
    if (fate(lo) != -1 || fate(hi) != 1) return 0.0;
    for (int it = 0; it < 64; ++it) {
        double mid = 0.5 * (lo + hi);
        if (fate(mid) == 1) hi = mid;
        else lo = mid;
    }
    return 0.5 * (lo + hi);
}

}  // namespace

extern "C" {

int so_shot_load(const char* ini_path, const char* const* overrides, int n_overrides, so_shot** out) {
    if (!out || !ini_path || n_overrides < 0 || (n_overrides > 0 && !overrides)) {
        so::set_global_error("so_shot_load: NULL path / output or bad override list");
        if (out) *out = nullptr;
        return SO_ERR_ARG;
    }
    *out = nullptr;
    so_shot* sh = new so_shot;
    std::string err;
    if (!sh->cfg.load(ini_path, &err)) {
        std::fprintf(stderr, "so_shot_load: %s\n", err.c_str());
        so::set_global_error("so_shot_load: " + err);
        delete sh;
        return SO_ERR_CONFIG;
    }
    for (int i = 0; i < n_overrides; ++i) {
        std::string kv = overrides[i] ? overrides[i] : "";
        size_t eq = kv.find('=');
        if (eq == std::string::npos) {
            so::set_global_error("so_shot_load: override '" + kv + "' is not key=value");
            delete sh;
            return SO_ERR_ARG;
        }
        sh->cfg.kv[trim(kv.substr(0, eq))] = trim(kv.substr(eq + 1));
    }
    build_scene(sh, &err);
    build_frames(sh);
    // Zoom target on the critical curve (main.cpp:421-428)
    if (sh->type == "render" && sh->cfg.has("camera.target_psi_deg")) {
        double psi = sh->cfg.num("camera.target_psi_deg", 0) * PI / 180;
        double rho = find_critical(sh, sh->frames[0], sh->S.a, psi) + sh->cfg.num("camera.target_offset_m", 0.0);
        sh->target_x = rho * std::cos(psi);
        sh->target_y = rho * std::sin(psi);
    }
    *out = sh;
    return SO_OK;
}

int so_shot_scene(const so_shot* s, so_scene* scene, so_tables* tables, so_scene_info* info) {
    if (!s) return SO_ERR_ARG;
    if (scene) *scene = s->S;
    if (tables) {
        tables->disk_lnT = s->disk_lnT.data();
        tables->disk_n = (int)s->disk_lnT.size();
        tables->k2_ln = s->k2_ln.data();
        tables->k2_n = (int)s->k2_ln.size();
        tables->bb_xyz = s->bb_xyz.data();
        tables->bb_n = (int)s->bb_xyz.size() / 3;
    }
    if (info) *info = s->info;
    return SO_OK;
}

int so_shot_settings(const so_shot* s, so_settings* rs) {
    if (!s || !rs) return SO_ERR_ARG;
    rs->W = s->cfg.integer("camera.width", 1920);
    rs->H = s->cfg.integer("camera.height", 1080);
    rs->spp = s->cfg.integer("render.spp", 8);
    rs->spp_max = s->cfg.integer("render.spp_max", 128);
    rs->target_err = (float)s->cfg.num("render.target_error", 0.03);
    return SO_OK;
}

int so_shot_nframes(const so_shot* s) { return s ? (int)s->frames.size() : 0; }

int so_shot_frame(const so_shot* s, int i, int W, uint32_t seed, so_frame* f) {
    if (!s || !f || i < 0 || i >= (int)s->frames.size() || W <= 0) return SO_ERR_ARG;
    *f = make_frame(s, s->frames[i], s->S.a, W, seed);
    return SO_OK;
}

int so_find_critical_point(const so_shot* s, int i, double a, double psi, double* rho) {
    if (!s || !rho || i < 0 || i >= (int)s->frames.size()) return SO_ERR_ARG;
    *rho = find_critical(s, s->frames[i], a, psi);
    return SO_OK;
}

int so_shot_get(const so_shot* s, const char* key, char* buf, int buflen) {
    if (!s || !key || !buf || buflen <= 0) return SO_ERR_ARG;
    if (!s->cfg.has(key)) return SO_ERR_CONFIG;
    std::snprintf(buf, (size_t)buflen, "%s", s->cfg.str(key).c_str());
    return SO_OK;
}

void so_shot_free(so_shot* s) { delete s; }

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
