// ref_gpu_harness.cpp -- TEST INFRASTRUCTURE ONLY.
//
// Drives the reference's own CUDA renderer (blackholes/src/render.cu, compiled unmodified from the
// reference sources by oracle/Makefile into _ref/libbhref_gpu.so) through the reference's own shot
// builders (common/config.cpp, blackholes/src/scene_build.cpp, shot.cpp, colour.cpp), the way its
// main program does (main.cpp:385-431 for the shot, :529 for each frame's seed), so that tests can
// render one frame through the reference and through this library on the same GPU and compare the
// images and the times.  No product code loads this library.
#include <cstdio>
#include <cstring>
#include <string>

#include "config.hpp"
#include "renderer.hpp"
#include "scene_build.hpp"
#include "shot.hpp"

namespace {
struct RefGpu {
    Config cfg;
    SceneGPU S{};
    SceneTables T;
    SceneInfo si;
    Shot shot;
    RenderSettings rs;
    Renderer R;
};

void put_error(char* buf, int len, const std::string& msg) {
    if (buf && len > 0) std::snprintf(buf, (size_t)len, "%s", msg.c_str());
}
}  // namespace

extern "C" {

// Loads the shot with "section.key=value" overrides, builds its scene and frames, finds the zoom
// target on the critical curve if the shot asks for one, and initialises the reference's Renderer
// on `device` (no star map).  NULL on failure, with the reason in err.
void* refgpu_open(const char* ini, const char* const* overrides, int n, int device, char* err, int errlen) {
    RefGpu* g = new RefGpu;
    std::string e;
    if (!g->cfg.load(ini, &e)) {
        put_error(err, errlen, e);
        delete g;
        return nullptr;
    }
    for (int i = 0; i < n; ++i) {
        std::string kv = overrides[i];
        size_t eq = kv.find('=');
        if (eq != std::string::npos) g->cfg.set(trim(kv.substr(0, eq)), trim(kv.substr(eq + 1)));
    }
    if (!build_scene(g->cfg, &g->S, &g->T, &g->si, &e) || !build_shot(g->cfg, &g->shot, &e)) {
        put_error(err, errlen, e);
        delete g;
        return nullptr;
    }
    g->rs.W = g->cfg.integer("camera.width", 1920);
    g->rs.H = g->cfg.integer("camera.height", 1080);
    g->rs.spp = g->cfg.integer("render.spp", 8);
    g->rs.spp_max = g->cfg.integer("render.spp_max", 128);
    g->rs.target_err = (float)g->cfg.num("render.target_error", 0.03);
    if (g->shot.type == "render" && g->cfg.has("camera.target_psi_deg")) {
        const double psi = g->cfg.num("camera.target_psi_deg", 0) * PI / 180;
        const double rho =
            find_critical_point(g->shot, g->shot.frames[0], g->S.a, psi) + g->cfg.num("camera.target_offset_m", 0.0);
        g->shot.target_x = rho * std::cos(psi);
        g->shot.target_y = rho * std::sin(psi);
    }
    if (!g->R.init(device, g->S, g->T, nullptr, g->rs, &e)) {
        put_error(err, errlen, e);
        delete g;
        return nullptr;
    }
    return g;
}

int refgpu_size(void* h, int* W, int* H, int* nframes) {
    const RefGpu* g = static_cast<RefGpu*>(h);
    *W = g->rs.W;
    *H = g->rs.H;
    *nframes = (int)g->shot.frames.size();
    return 0;
}

// Frame i through Renderer::render (pass 1, the adaptive pass when spp_max > spp, resolve; no post
// filter), its HDR pixels (W * H * 4 floats) into px, the renderer's own trace time (ms_trace: host
// clock around the synchronous trace) and sample counters.
int refgpu_render(void* h, int i, float* px, double* ms_trace, long long* samples, long long* step_limited) {
    RefGpu* g = static_cast<RefGpu*>(h);
    if (i < 0 || i >= (int)g->shot.frames.size()) return 1;
    const FrameGPU F = make_frame(g->shot, g->shot.frames[(size_t)i], g->S.a, g->rs.W, 0x9E3779B9u * (uint32_t)(i + 1));
    PostParams pp;
    HdrFrame out;
    RenderStats st;
    g->R.render(F, pp, 0.995, &out, &st);
    std::memcpy(px, out.px.data(), out.px.size() * sizeof(float));
    if (ms_trace) *ms_trace = st.ms_trace;
    if (samples) *samples = st.samples;
    if (step_limited) *step_limited = st.step_limited;
    return 0;
}

void refgpu_close(void* h) { delete static_cast<RefGpu*>(h); }

}  // extern "C"
