// so_shot.cpp -- shot files -> so_scene, its tables, and so_frame per frame (host side of the boundary).
//
// A shot is the reference's .ini: the file format of common/config.cpp:14-63, the scene keys and
// defaults of blackholes/src/scene_build.cpp:83-213, the frames and camera tracks of
// blackholes/src/shot.cpp:73-146, the --set overrides and critical-curve zoom target of
// blackholes/src/main.cpp:389-428; plus this library's [so] keys (torus plasma, read by the callers).
// Shots drop in unchanged and give the reference's structs bit for bit.  The pieces:
//   KeyValues     the file as flat "section.key" -> value text;
//   kSceneSchema  one row per plain scene parameter: key, default, unit factor, so_scene field, storage;
//   build_scene   the schema interpreter, then what depends on other values (spin clamp, horizon and
//                 ISCO, units, seed, tables from so_scene_tables.cpp, the sky rotation);
//   Track         one animated parameter: knots with monotone cubic Hermite tangents (Fritsch &
//                 Carlson 1980, weighted-harmonic-mean form of Fritsch & Butland 1984), flat at the ends,
//                 optionally in log space;
//   kPathSchema   the per-frame camera parameters, each a constant or a track;
//   frame_of      so_frame of one frame: camera basis by Rodrigues rotations, pixel scale, zoom target,
//                 orbiting-camera boost.
// Host code is compiled with -ffp-contract=off: each expression below rounds as it is written.
#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <string>
#include <vector>

#include "so_kerr.cuh"
#include "so_scene_tables.h"

namespace so {
namespace {

constexpr double kDeg = PI / 180;  // degrees -> radians for the per-frame camera angles

std::string trim(const std::string& s) {
    const char* ws = " \t\r\n";
    const size_t a = s.find_first_not_of(ws);
    return a == std::string::npos ? std::string() : s.substr(a, s.find_last_not_of(ws) - a + 1);
}

// Text before any '#', trimmed.
std::string strip_comment(const std::string& s) { return trim(s.substr(0, s.find('#'))); }

// ---- the .ini as key/value text ------------------------------------------------------------------
class KeyValues {
  public:
    // Reads `path` into the store: [section] headers, key = value lines (stored as section.key),
    // '#' comments, a trailing '\' joining the next line, and a top-level `include = file` that reads
    // that file (relative to the including one) at that point, so later keys override it.
    bool read(const std::string& path, std::string* err) {
        std::ifstream in(path);
        if (!in) {
            *err = "cannot open " + path;
            return false;
        }
        std::vector<std::string> lines;
        for (std::string s; std::getline(in, s);) lines.push_back(s);
        const size_t slash = path.find_last_of('/');
        const std::string dir = slash == std::string::npos ? "." : path.substr(0, slash);
        std::string section;
        for (size_t next = 0; next < lines.size();) {
            std::string line = strip_comment(lines[next++]);
            while (!line.empty() && line.back() == '\\' && next < lines.size()) {
                line.pop_back();
                line = trim(line + " " + strip_comment(lines[next++]));
            }
            const std::string where = path + ":" + std::to_string(next) + ": ";
            if (line.empty()) continue;
            if (line.front() == '[') {
                if (line.back() != ']') {
                    *err = where + "bad section header";
                    return false;
                }
                section = trim(line.substr(1, line.size() - 2));
                continue;
            }
            const size_t eq = line.find('=');
            if (eq == std::string::npos) {
                *err = where + "expected key = value";
                return false;
            }
            const std::string key = trim(line.substr(0, eq)), value = trim(line.substr(eq + 1));
            if (section.empty() && key == "include") {
                if (value.empty()) {
                    *err = where + "empty include";
                    return false;
                }
                if (!read(value.front() == '/' ? value : dir + "/" + value, err)) return false;
                continue;
            }
            kv_[section.empty() ? key : section + "." + key] = value;
        }
        return true;
    }
    void set(const std::string& key, const std::string& value) { kv_[key] = value; }
    bool has(const std::string& key) const { return kv_.count(key) != 0; }
    const std::string* find(const std::string& key) const {
        const auto it = kv_.find(key);
        return it == kv_.end() ? nullptr : &it->second;
    }
    std::string text(const std::string& key, const std::string& fallback = "") const {
        const std::string* v = find(key);
        return v ? *v : fallback;
    }
    // A number: the leading number of the value, or `fallback` if the key is missing, empty or
    // does not start with a number.
    double real(const std::string& key, double fallback) const {
        const std::string* v = find(key);
        if (!v || v->empty()) return fallback;
        char* end = nullptr;
        const double x = std::strtod(v->c_str(), &end);
        return end == v->c_str() ? fallback : x;
    }
    int whole(const std::string& key, int fallback) const { return (int)real(key, fallback); }
    // A switch: 1/true/yes/on or 0/false/no/off; anything else leaves `fallback`.
    bool truth(const std::string& key, bool fallback) const {
        const std::string* v = find(key);
        if (!v) return fallback;
        static const char* const kOn[] = {"1", "true", "yes", "on"};
        static const char* const kOff[] = {"0", "false", "no", "off"};
        for (const char* w : kOn)
            if (*v == w) return true;
        for (const char* w : kOff)
            if (*v == w) return false;
        return fallback;
    }

  private:
    std::map<std::string, std::string> kv_;
};

// ---- the scene schema --------------------------------------------------------------------------
enum class Store : unsigned char { F64, F32, I32, Switch, SwitchF32 };
enum class OnBy : unsigned char { Never, Always, Visible, Radio };  // default state of a switch

struct SceneParam {
    const char* key;
    double fallback;  // default value (numbers)
    double unit;      // factor applied to the number read
    Store store;
    size_t offset;    // field in so_scene
    OnBy on;          // default of a switch
};

#define SO_AT(field) offsetof(so_scene, field)
const SceneParam kSceneSchema[] = {
    {"render.tolerance", 1e-9, 1.0, Store::F64, SO_AT(tol), OnBy::Never},
    {"render.max_steps", 20000, 1.0, Store::I32, SO_AT(max_steps), OnBy::Never},
    {"render.r_escape", 2e4, 1.0, Store::F64, SO_AT(r_escape), OnBy::Never},
    {"render.step_fraction", 0.04, 1.0, Store::F64, SO_AT(step_frac), OnBy::Never},
    // thin disk
    {"disk.enabled", 0, 1.0, Store::Switch, SO_AT(disk_on), OnBy::Visible},
    {"disk.r_out", 40.0, 1.0, Store::F64, SO_AT(disk_rout), OnBy::Never},
    {"disk.turbulence", 0.45, 1.0, Store::F32, SO_AT(disk_turb_amp), OnBy::Never},
    {"disk.turbulence_scale", 0.35, 1.0, Store::F32, SO_AT(disk_turb_scale), OnBy::Never},
    {"disk.correlation_orbits", 0.6, 1.0, Store::F32, SO_AT(disk_tcorr), OnBy::Never},
    {"disk.limb_darkening", 0, 1.0, Store::SwitchF32, SO_AT(disk_ld), OnBy::Always},
    {"disk.color_correction", 1.0, 1.0, Store::F32, SO_AT(disk_fcol), OnBy::Never},
    // hot flow
    {"flow.enabled", 0, 1.0, Store::Switch, SO_AT(flow_on), OnBy::Radio},
    {"flow.n0", 1e5, 1.0, Store::F64, SO_AT(n0), OnBy::Never},
    {"flow.n_index", 1.1, 1.0, Store::F64, SO_AT(n_index), OnBy::Never},
    {"flow.theta0", 25.0, 1.0, Store::F64, SO_AT(theta0), OnBy::Never},
    {"flow.theta_index", 0.84, 1.0, Store::F64, SO_AT(theta_index), OnBy::Never},
    {"flow.h_over_r", 0.4, 1.0, Store::F64, SO_AT(h_r), OnBy::Never},
    {"flow.beta", 10.0, 1.0, Store::F64, SO_AT(beta_p), OnBy::Never},
    {"flow.r_max", 60.0, 1.0, Store::F64, SO_AT(r_flow_max), OnBy::Never},
    {"flow.nu_ghz", 230.0, 1e9, Store::F64, SO_AT(nu_obs), OnBy::Never},  // stored in Hz
    {"flow.keplerian_fraction", 0.9, 1.0, Store::F64, SO_AT(flow_kep), OnBy::Never},
    {"flow.turbulence", 0.7, 1.0, Store::F32, SO_AT(flow_turb_amp), OnBy::Never},
    {"flow.turbulence_scale", 0.45, 1.0, Store::F32, SO_AT(flow_turb_scale), OnBy::Never},
    {"flow.correlation_orbits", 0.5, 1.0, Store::F32, SO_AT(flow_tcorr), OnBy::Never},
    // star map
    {"sky.enabled", 0, 1.0, Store::Switch, SO_AT(sky_on), OnBy::Visible},
    {"sky.brightness", 1.0, 1.0, Store::F32, SO_AT(sky_scale), OnBy::Never},
};
#undef SO_AT

void apply_schema(const KeyValues& kv, int mode, so_scene* S) {
    unsigned char* base = reinterpret_cast<unsigned char*>(S);
    for (const SceneParam& p : kSceneSchema) {
        unsigned char* dst = base + p.offset;
        const bool on_by_default = p.on == OnBy::Always || (p.on == OnBy::Visible && mode == SO_MODE_VISIBLE) ||
                                   (p.on == OnBy::Radio && mode == SO_MODE_RADIO);
        switch (p.store) {
            case Store::F64: {
                const double v = kv.real(p.key, p.fallback) * p.unit;
                std::memcpy(dst, &v, sizeof v);
                break;
            }
            case Store::F32: {
                const float v = (float)(kv.real(p.key, p.fallback) * p.unit);
                std::memcpy(dst, &v, sizeof v);
                break;
            }
            case Store::I32: {
                const int v = (int)(kv.real(p.key, p.fallback) * p.unit);
                std::memcpy(dst, &v, sizeof v);
                break;
            }
            case Store::Switch: {
                const int v = kv.truth(p.key, on_by_default) ? 1 : 0;
                std::memcpy(dst, &v, sizeof v);
                break;
            }
            case Store::SwitchF32: {
                const float v = kv.truth(p.key, on_by_default) ? 1.f : 0.f;
                std::memcpy(dst, &v, sizeof v);
                break;
            }
        }
    }
}

// ---- small vector algebra for the camera and sky frames ----------------------------------------
struct V3 {
    double x, y, z;
};
V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
V3 operator-(V3 a) { return {-a.x, -a.y, -a.z}; }
V3 operator*(V3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
V3 cross(V3 a, V3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
double norm(V3 a) { return std::sqrt(dot(a, a)); }
V3 unit(V3 a) { return a * (1.0 / norm(a)); }
double comp(V3 a, int i) { return i == 0 ? a.x : i == 1 ? a.y : a.z; }
so_vec3 to_abi(V3 a) { return so_vec3{a.x, a.y, a.z}; }
// v turned by `angle` about the unit vector `axis` (Rodrigues' formula)
V3 rotated(V3 v, V3 axis, double angle) {
    const double c = std::cos(angle), s = std::sin(angle);
    return v * c + cross(axis, v) * s + axis * (dot(axis, v) * (1 - c));
}

// Rotation from the hole's frame to galactic coordinates: the direction straight behind the hole, as
// seen by a camera at inclination `incl` and azimuth `phi`, goes to galactic (l, b), its projected
// spin axis to the galactic north turned by `roll` about that direction.  Rows of
// M = g_behind behind^T + g_up up^T + g_side side^T.
so_mat3 sky_rotation(double incl, double phi, double l, double b, double roll) {
    const V3 z = {0, 0, 1};
    const V3 behind = -V3{std::sin(incl) * std::cos(phi), std::sin(incl) * std::sin(phi), std::cos(incl)};
    V3 up = unit(z - behind * dot(z, behind));
    if (!(norm(up) > 0.5)) up = {1, 0, 0};  // camera on the axis
    const V3 side = cross(up, behind);
    const V3 g_behind = {std::cos(b) * std::cos(l), std::cos(b) * std::sin(l), std::sin(b)};
    const V3 g_north = unit(z - g_behind * dot(z, g_behind));
    const V3 g_east = cross(g_north, g_behind);
    const V3 g_up = g_north * std::cos(roll) + g_east * std::sin(roll);
    const V3 g_side = cross(g_up, g_behind);
    V3 row[3];
    for (int i = 0; i < 3; ++i)
        row[i] = V3{comp(g_behind, i) * behind.x + comp(g_up, i) * up.x + comp(g_side, i) * side.x,
                    comp(g_behind, i) * behind.y + comp(g_up, i) * up.y + comp(g_side, i) * side.y,
                    comp(g_behind, i) * behind.z + comp(g_up, i) * up.z + comp(g_side, i) * side.z};
    return so_mat3{to_abi(row[0]), to_abi(row[1]), to_abi(row[2])};
}

// ---- animated parameters -----------------------------------------------------------------------
class Track {
  public:
    // "time:value, time:value, ..." (times in seconds of the shot); false if an entry has no ':' or
    // the list is empty.
    static bool parse(const std::string& text, bool log_space, Track* out) {
        Track tr;
        tr.log_ = log_space;
        size_t pos = 0;
        while (pos <= text.size()) {
            const size_t comma = std::min(text.find(',', pos), text.size());
            const std::string item = trim(text.substr(pos, comma - pos));
            pos = comma + 1;
            if (item.empty()) continue;
            const size_t colon = item.find(':');
            if (colon == std::string::npos) return false;
            const double v = std::strtod(item.substr(colon + 1).c_str(), nullptr);
            tr.t_.push_back(std::strtod(item.substr(0, colon).c_str(), nullptr));
            tr.v_.push_back(log_space ? std::log(v) : v);
        }
        if (tr.t_.empty()) return false;
        tr.tangents();
        *out = tr;
        return true;
    }

    double at(double time) const {
        const size_t n = t_.size();
        double out;
        if (n == 1 || time <= t_[0]) {
            out = v_[0];
        } else if (time >= t_[n - 1]) {
            out = v_[n - 1];
        } else {
            // the first knot at or after `time` (among the inner knots) ends the interval
            const size_t k = (size_t)(std::find_if(t_.begin() + 1, t_.end() - 1, [&](double tk) { return time <= tk; }) -
                                      t_.begin()) - 1;
            const double h = t_[k + 1] - t_[k], s = (time - t_[k]) / h;
            // cubic Hermite basis on [0, 1]
            const double b00 = (1 + 2 * s) * (1 - s) * (1 - s), b10 = s * (1 - s) * (1 - s), b01 = s * s * (3 - 2 * s),
                         b11 = s * s * (s - 1);
            out = b00 * v_[k] + b10 * h * m_[k] + b01 * v_[k + 1] + b11 * h * m_[k + 1];
        }
        return log_ ? std::exp(out) : out;
    }

  private:
    // Fritsch-Carlson tangents: zero at the end knots and at local extrema, elsewhere the weighted
    // harmonic mean of the neighbouring secants, which keeps each interval monotone.
    void tangents() {
        const size_t n = t_.size();
        m_.assign(n, 0.0);
        for (size_t k = 1; k + 1 < n; ++k) {
            const double h0 = t_[k] - t_[k - 1], h1 = t_[k + 1] - t_[k];
            const double d0 = (v_[k] - v_[k - 1]) / h0, d1 = (v_[k + 1] - v_[k]) / h1;
            if (d0 * d1 <= 0) continue;
            m_[k] = 3.0 * (h0 + h1) / ((2.0 * h1 + h0) / d0 + (h1 + 2.0 * h0) / d1);
        }
    }
    std::vector<double> t_, v_, m_;
    bool log_ = false;
};

// ---- per-frame camera parameters ---------------------------------------------------------------
struct CameraState {
    double t = 0, r = 0, incl = 0, phi = 0, roll = 0, yaw = 0, pitch = 0, fov = 0;
    bool fov_in_m = false;
    double zoom = 1, target = 0, off_x = 0, off_y = 0, time_m = 0;
};

struct PathParam {
    const char* key;
    double fallback;
    bool log_space;  // tracks interpolate ln(value)
    double unit;     // factor applied to the value (degrees -> radians)
    double CameraState::*field;
};
const PathParam kPathSchema[] = {
    {"camera.r", 1e6, true, 1.0, &CameraState::r},
    {"camera.incl", 80, false, kDeg, &CameraState::incl},
    {"camera.phi", 0, false, kDeg, &CameraState::phi},
    {"camera.roll", 0, false, kDeg, &CameraState::roll},
    {"camera.yaw", 0, false, kDeg, &CameraState::yaw},
    {"camera.pitch", 0, false, kDeg, &CameraState::pitch},
    {"camera.zoom", 1, true, 1.0, &CameraState::zoom},
    {"camera.target", 0, false, 1.0, &CameraState::target},
    {"camera.offset_x_m", 0, false, 1.0, &CameraState::off_x},
    {"camera.offset_y_m", 0, false, 1.0, &CameraState::off_y},
    {"time.t_m", 0, false, 1.0, &CameraState::time_m},
};

// A parameter at shot time `t`: its track ("track.<key>") where one parses, else its constant.
double path_value(const KeyValues& kv, const char* key, double fallback, bool log_space, double t) {
    const std::string* track_text = kv.find(std::string("track.") + key);
    Track tr;
    if (track_text && Track::parse(*track_text, log_space, &tr)) return tr.at(t);
    return kv.real(key, fallback);
}

}  // namespace

// Scene scalars of the vacuum geodesics for spin a (the scene builder's clamp, horizon, ISCO and
// stopping radius with the same horizon margin); the tables and the emitters' parameters stay.
void scene_set_spin(so_scene* S, double a) {
    const double margin = S->r_stop - S->rh;
    if (a <= 0.0) a = 1e-6;
    if (a > 0.9999) a = 0.9999;
    S->a = a;
    S->rh = horizon_radius(a);
    S->r_isco = tables::isco(a);
    S->r_stop = S->rh + margin;
}

void set_global_error(const std::string& msg);  // so_renderer.cpp: so_last_error(NULL)
}  // namespace so

using namespace so;

struct so_shot {
    KeyValues kv;
    so_scene S;
    so_scene_info info;
    std::vector<float> disk_lnT, k2_ln, bb_xyz;
    std::string name, type, motion;
    double duration = 5, fps = 30, target_x = 0, target_y = 0;
    std::vector<CameraState> frames;
};

namespace {

void build_scene(so_shot* sh) {
    const KeyValues& kv = sh->kv;
    so_scene* S = &sh->S;
    so_scene_info& info = sh->info;
    std::memset(S, 0, sizeof(so_scene));
    std::memset(&info, 0, sizeof info);

    S->mode = kv.text("render.mode", "visible") == "radio" ? SO_MODE_RADIO : SO_MODE_VISIBLE;
    apply_schema(kv, S->mode, S);

    // Spin: the orbit formulas divide by a, so a = 0 becomes 1e-6 (Schwarzschild to that accuracy);
    // the largest spin is 0.9999.
    double a = kv.real("bh.spin", 0.94);
    a = a <= 0.0 ? 1e-6 : std::min(a, 0.9999);
    S->a = a;
    S->rh = horizon_radius(a);
    S->r_isco = tables::isco(a);
    S->r_stop = S->rh + kv.real("render.horizon_margin", 0.01);
    S->disk_rin = std::max(kv.real("disk.r_in", 0.0), S->r_isco);
    S->seed = (uint32_t)kv.whole("render.seed", 1) * 2654435761u;  // Knuth's multiplicative hash

    // Physical scale (cgs, CODATA / IAU values)
    const double parsec = 3.0856775814913673e18, grav = 6.67430e-8, m_sun = 1.98847e33, c_cgs = 2.99792458e10;
    info.mass_msun = kv.real("bh.mass_msun", 6.5e9);
    const double distance_pc =
        kv.has("bh.distance_mpc") ? kv.real("bh.distance_mpc", 16.8) * 1e6 : kv.real("bh.distance_pc", 16.8e6);
    info.distance_cm = distance_pc * parsec;
    info.rg_cm = grav * info.mass_msun * m_sun / (c_cgs * c_cgs);
    info.tg_s = info.rg_cm / c_cgs;
    info.uas_per_m = info.rg_cm / info.distance_cm * (180.0 / PI * 3600.0e6);
    info.radio_flux_target_jy = kv.real("flow.flux_jy", 0.0);
    S->rg_cm = info.rg_cm;

    // Novikov-Thorne disk temperature (peak from the Eddington ratio unless disk.t_max is given)
    const tables::DiskProfile disk = tables::disk_profile(a, S->r_isco, S->disk_rout, info.mass_msun, info.rg_cm,
                                                          kv.real("disk.eddington_ratio", 0.1));
    info.disk_tmax = kv.real("disk.t_max", disk.t_max_physical);
    info.disk_mdot_edd = disk.eddington_at(info.disk_tmax);
    sh->disk_lnT = disk.ln_temperature(info.disk_tmax);
    S->disk_n = tables::DiskProfile::kSize;
    S->disk_lr0 = disk.ln_r0;
    S->disk_dlr = disk.dln_r;

    // ln K2 of the electron temperature, Theta_e in [0.02, 1e4]
    sh->k2_ln = tables::ln_bessel_k2_table(512, 0.02, 1e4, &S->k2_l0, &S->k2_dl);
    S->k2_n = 512;

    S->sky_rot = sky_rotation(kv.real("camera.incl", 80.0) * PI / 180, kv.real("camera.phi", 0.0) * PI / 180,
                              kv.real("sky.l_deg", 0.0) * PI / 180, kv.real("sky.b_deg", 0.0) * PI / 180,
                              kv.real("sky.roll_deg", 0.0) * PI / 180);

    sh->bb_xyz = tables::blackbody_xyz_table(&S->bb_l0, &S->bb_dl);
    S->bb_n = tables::kBlackbodyN;
    S->disk_lnT = sh->disk_lnT.data();
    S->k2_lntab = sh->k2_ln.data();
    S->bb_xyz = sh->bb_xyz.data();
}

void build_frames(so_shot* sh) {
    const KeyValues& kv = sh->kv;
    sh->name = kv.text("shot.name", "shot");
    sh->type = kv.text("shot.type", "render");
    sh->duration = kv.real("shot.duration", 5);
    sh->fps = kv.real("shot.fps", 30);
    sh->motion = kv.text("camera.motion", "static");
    int n = std::max(1, (int)std::lround(sh->duration * sh->fps));
    if (kv.has("shot.frames")) n = kv.whole("shot.frames", n);
    const bool fov_in_m = kv.has("camera.fov_m") || kv.has("track.camera.fov_m");
    sh->frames.assign((size_t)std::max(n, 0), CameraState());
    for (int i = 0; i < n; ++i) {
        CameraState& st = sh->frames[(size_t)i];
        st.t = i / sh->fps;
        for (const PathParam& p : kPathSchema)
            st.*p.field = path_value(kv, p.key, p.fallback, p.log_space, st.t) * p.unit;
        st.fov_in_m = fov_in_m;
        st.fov = fov_in_m ? path_value(kv, "camera.fov_m", 30, true, st.t)
                          : path_value(kv, "camera.fov_deg", 40, true, st.t) * kDeg;
    }
}

so_frame frame_of(const so_shot* sh, const CameraState& st, double a, int W, uint32_t seed) {
    so_frame F;
    std::memset(&F, 0, sizeof F);
    F.r = st.r;
    F.th = st.incl;
    F.ph = st.phi;
    F.t = st.time_m;
    kerr_point(a, st.r, st.incl, &F.kp);
    // Camera basis in the ZAMO frame (e_r, e_theta, e_phi), looking at the hole: forward = -e_r,
    // up = -e_theta (towards the spin axis), right = e_phi; then yaw about up, pitch about right,
    // roll about forward.
    V3 fwd = {-1, 0, 0}, up = {0, -1, 0}, right = {0, 0, 1};
    if (st.yaw != 0) {
        fwd = rotated(fwd, up, -st.yaw);
        right = rotated(right, up, -st.yaw);
    }
    if (st.pitch != 0) {
        fwd = rotated(fwd, right, st.pitch);
        up = rotated(up, right, st.pitch);
    }
    if (st.roll != 0) {
        right = rotated(right, fwd, st.roll);
        up = rotated(up, fwd, st.roll);
    }
    F.F = to_abi(fwd);
    F.R = to_abi(right);
    F.U = to_abi(up);
    // Tangent-plane width: a field of view in M at the camera's distance, or an angle
    const double width = st.fov_in_m ? st.fov / st.r : 2.0 * std::tan(0.5 * st.fov);
    F.pix = width / st.zoom / W;
    if (st.fov_in_m) {
        F.cx = (st.off_x + st.target * sh->target_x) / st.r;
        F.cy = (st.off_y + st.target * sh->target_y) / st.r;
    }
    if (sh->motion == "orbit") {
        // circular Keplerian orbit of the camera: its speed relative to the ZAMO, capped at 0.98 c
        const double omega_k = 1.0 / (std::pow(st.r, 1.5) + a);
        const double v = (omega_k - F.kp.omega) * F.kp.e_psi / F.kp.e_nu;
        F.beta = so_vec3{0, 0, std::max(-0.98, std::min(0.98, v))};
    }
    F.seed = seed;
    return F;
}

// Image radius (M) of the critical curve at image angle psi: bisection between a captured ray at
// 0.5 M and an escaping one at 15 M on the vacuum fate (tolerance 1e-12, escape at 200 M), 64 halvings.
// 0 if the bracket does not hold.
double find_critical(const so_shot* sh, const CameraState& st, double a, double psi) {
    so_frame G = frame_of(sh, st, a, 1, 0);
    G.cx = 0;
    G.cy = 0;
    auto fate = [&](double rho) {
        const double x = rho * std::cos(psi) / st.r, y = rho * std::sin(psi) / st.r;
        return vacuum_fate(a, G, view_dir(G, x, y), 1e-12, 200.0, 2000000);
    };
    double inside = 0.5, outside = 15.0;
    if (fate(inside) != -1 || fate(outside) != 1) return 0.0;
    for (int it = 0; it < 64; ++it) {
        const double mid = 0.5 * (inside + outside);
        (fate(mid) == 1 ? outside : inside) = mid;
    }
    return 0.5 * (inside + outside);
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
    if (!sh->kv.read(ini_path, &err)) {
        std::fprintf(stderr, "so_shot_load: %s\n", err.c_str());
        so::set_global_error("so_shot_load: " + err);
        delete sh;
        return SO_ERR_CONFIG;
    }
    for (int i = 0; i < n_overrides; ++i) {  // --set section.key=value
        const std::string kv = overrides[i] ? overrides[i] : "";
        const size_t eq = kv.find('=');
        if (eq == std::string::npos) {
            so::set_global_error("so_shot_load: override '" + kv + "' is not key=value");
            delete sh;
            return SO_ERR_ARG;
        }
        sh->kv.set(trim(kv.substr(0, eq)), trim(kv.substr(eq + 1)));
    }
    build_scene(sh);
    build_frames(sh);
    // Zoom target on the critical curve at image angle camera.target_psi_deg, found for frame 0
    if (sh->type == "render" && sh->kv.has("camera.target_psi_deg") && !sh->frames.empty()) {
        const double psi = sh->kv.real("camera.target_psi_deg", 0) * PI / 180;
        const double rho =
            find_critical(sh, sh->frames[0], sh->S.a, psi) + sh->kv.real("camera.target_offset_m", 0.0);
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
    rs->W = s->kv.whole("camera.width", 1920);
    rs->H = s->kv.whole("camera.height", 1080);
    rs->spp = s->kv.whole("render.spp", 8);
    rs->spp_max = s->kv.whole("render.spp_max", 128);
    rs->target_err = (float)s->kv.real("render.target_error", 0.03);
    return SO_OK;
}

int so_shot_nframes(const so_shot* s) { return s ? (int)s->frames.size() : 0; }

int so_shot_frame(const so_shot* s, int i, int W, uint32_t seed, so_frame* f) {
    if (!s || !f || i < 0 || i >= (int)s->frames.size() || W <= 0) return SO_ERR_ARG;
    *f = frame_of(s, s->frames[(size_t)i], s->S.a, W, seed);
    return SO_OK;
}

int so_find_critical_point(const so_shot* s, int i, double a, double psi, double* rho) {
    if (!s || !rho || i < 0 || i >= (int)s->frames.size()) return SO_ERR_ARG;
    *rho = find_critical(s, s->frames[(size_t)i], a, psi);
    return SO_OK;
}

int so_shot_get(const so_shot* s, const char* key, char* buf, int buflen) {
    if (!s || !key || !buf || buflen <= 0) return SO_ERR_ARG;
    const std::string* v = s->kv.find(key);
    if (!v) return SO_ERR_CONFIG;
    std::snprintf(buf, (size_t)buflen, "%s", v->c_str());
    return SO_OK;
}

void so_shot_free(so_shot* s) { delete s; }

}  // extern "C"
