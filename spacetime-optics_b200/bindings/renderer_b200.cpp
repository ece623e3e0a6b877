// renderer_b200.cpp -- Renderer on top of libso_tracer.so (link with -lso_tracer)
#include "renderer.hpp"
#include "so_tracer.h"

static_assert(sizeof(SceneGPU) == sizeof(so_scene), "layout");
static_assert(sizeof(FrameGPU) == sizeof(so_frame), "layout");

struct Renderer::Impl { so_renderer* r = nullptr; RenderSettings rs; };

Renderer::Renderer() : p_(new Impl) {}
Renderer::~Renderer() { so_destroy(p_->r); delete p_; }

bool Renderer::init(int device, const SceneGPU& s, const SceneTables& T, const SkyTexture* sky,
                    const RenderSettings& rs, std::string* err) {
    so_tables t = {T.disk_lnT.data(), (int)T.disk_lnT.size(), T.k2_ln.data(), (int)T.k2_ln.size(),
                   T.bb_xyz.data(), (int)T.bb_xyz.size() / 3};
    so_settings st = {rs.W, rs.H, rs.spp, rs.spp_max, rs.target_err};
    p_->rs = rs;
    int rc = so_init(&p_->r, device, reinterpret_cast<const so_scene*>(&s), &t, &st);
    if (rc && err) *err = so_last_error(nullptr);
    if (rc == SO_OK && sky && sky->w > 0) rc = so_set_sky(p_->r, sky->w, sky->h, sky->data.data());
    if (rc && err && err->empty()) *err = so_last_error(p_->r);
    return rc == SO_OK;
}

void Renderer::update_scene(const SceneGPU& s) { so_update_scene(p_->r, reinterpret_cast<const so_scene*>(&s)); }

void Renderer::render(const FrameGPU& f, const PostParams& post, double pct, HdrFrame* out, RenderStats* st) {
    out->px.resize((size_t)p_->rs.W * p_->rs.H * 4);
    so_hdr_frame h = {0, 0, out->px.data(), 0, 0};
    so_post pp = {post.bloom, post.blur_sigma_px, post.hide_direct};   // glare / beam as the reference
    so_stats s{};
    if (so_render(p_->r, reinterpret_cast<const so_frame*>(&f), &pp, pct, &h, &s) != SO_OK)
        std::fprintf(stderr, "bhrt: %s\n", so_last_error(p_->r));
    out->W = h.W; out->H = h.H; out->lum_percentile = h.lum_percentile; out->lum_max = h.lum_max;
    if (st) { st->ms_trace = s.ms_trace; st->ms_post = s.ms_post; st->samples = s.samples; st->step_limited = s.step_limited; }
}

double Renderer::radio_flux(FrameGPU f, int n, double pix_sr) {
    double jy = 0;
    so_radio_flux(p_->r, reinterpret_cast<const so_frame*>(&f), n, pix_sr, &jy);
    return jy;
}
