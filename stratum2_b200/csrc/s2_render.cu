// Wavefront path tracer (placeholder until the kernels land).
#include "s2_context.h"

namespace s2 {
struct RenderState {};
void destroy_render_state(S2Context* ctx) { delete ctx->render; ctx->render = nullptr; }
}  // namespace s2

extern "C" void s2_default_render_params(S2RenderParams* p) {
    if (!p) return;
    *p = S2RenderParams{};
    p->min_path_length = 0;
    p->max_path_length = 5;
    p->exposure = 0.f;
    p->spp = 1;
    p->environment_sample_probability = 0.9f;
    p->restir_candidates = 32;
    p->restir_max_m = 3.f;
}

extern "C" int s2_render(S2Context* ctx, const S2View*, const S2RenderParams*, const S2Aovs*, int, S2RenderStats*) {
    return s2::set_error(ctx, S2_ERR_UNSUPPORTED, "render not built yet");
}
