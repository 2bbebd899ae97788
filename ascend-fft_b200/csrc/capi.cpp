// extern "C" layer over bfly::Context / bfly::Plan (declarations in include/bfly_b200.h).
#include "bfly_b200.h"

#include "bfly/plan.hpp"

#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

struct bfly_context {
    bfly::Context ctx;
};
struct bfly_plan {
    std::unique_ptr<bfly::Plan> plan;
};
struct bfly_ragged {
    std::unique_ptr<bfly::Ragged> ragged;
};

namespace {
int copyOut(const std::string& s, char* buf, size_t cap, size_t* needed) {
    if (needed) *needed = s.size() + 1;
    if (!buf || !cap) return 0;
    const size_t n = s.size() < cap - 1 ? s.size() : cap - 1;
    std::memcpy(buf, s.data(), n);
    buf[n] = 0;
    return s.size() + 1 > cap ? -11 : 0;
}

}  // namespace

extern "C" {

const char* bfly_version(void) { return "bfly_b200 0.1.0 (sm_100a)"; }

int bfly_context_create(bfly_context** out) {
    if (!out) return -10;
    *out = new (std::nothrow) bfly_context;
    return *out ? 0 : -3;
}

void bfly_context_destroy(bfly_context* ctx) { delete ctx; }

int bfly_context_init(bfly_context* ctx, const char* profile_path, const char* space_path,
                      const char* kernel_path) {
    if (!ctx || !profile_path || !space_path) return -10;
    return ctx->ctx.init(profile_path, space_path, kernel_path ? kernel_path : "builtin");
}

int bfly_context_init_device(bfly_context* ctx, const char* profile_path, const char* space_path,
                             const char* kernel_path, int device) {
    if (!ctx || !profile_path || !space_path) return -10;
    return ctx->ctx.init(profile_path, space_path, kernel_path ? kernel_path : "builtin", device);
}

int bfly_context_enumerate(bfly_context* ctx, uint32_t n, uint32_t batch, char* buf, size_t cap,
                           int* count, size_t* needed) {
    if (!ctx) return -10;
    const auto cs = ctx->ctx.enumerate(n, batch);
    std::string s;
    for (const auto& c : cs) {
        s += c.id;
        s += '\t';
        s += bfly::toString(c.state);
        s += '\t';
        s += c.reason;
        s += '\n';
    }
    if (count) *count = (int)cs.size();
    return copyOut(s, buf, cap, needed);
}

int bfly_context_select(bfly_context* ctx, uint32_t n, uint32_t batch, int top_k, bfly_plan** out,
                        char* log, size_t log_cap) {
    if (!ctx || !out) return -10;
    *out = nullptr;
    std::string text;
    auto p = ctx->ctx.select(n, batch, top_k, log ? &text : nullptr);
    if (log) copyOut(text, log, log_cap, nullptr);
    if (!p) return -1;
    *out = new bfly_plan{std::move(p)};
    return 0;
}

int bfly_context_make_plan(bfly_context* ctx, uint32_t n, uint32_t batch, const char* candidate_id,
                           bfly_plan** out) {
    if (!ctx || !out || !candidate_id) return -10;
    *out = nullptr;
    for (const auto& c : ctx->ctx.enumerate(n, batch)) {
        if (c.id != candidate_id) continue;
        auto p = ctx->ctx.makePlan(c);
        if (!p) return -1;
        *out = new bfly_plan{std::move(p)};
        return 0;
    }
    return -8;
}

int bfly_context_set_tuning_cache(bfly_context* ctx, const char* path) {
    if (!ctx) return -10;
    ctx->ctx.setTuningCache(path ? path : "");
    return 0;
}

void* bfly_context_stream(bfly_context* ctx) { return ctx ? ctx->ctx.stream() : nullptr; }

void bfly_plan_destroy(bfly_plan* plan) { delete plan; }

int bfly_plan_candidate_id(bfly_plan* plan, char* buf, size_t cap) {
    if (!plan || !plan->plan) return -10;
    return copyOut(plan->plan->candidate().id, buf, cap, nullptr);
}

#define PLAN_OR_FAIL()                  \
    if (!plan || !plan->plan) return -10; \
    bfly::Plan& p = *plan->plan

int bfly_plan_prepare(bfly_plan* plan, uint32_t n, uint32_t batch) {
    PLAN_OR_FAIL();
    return p.prepare(n, batch);
}

int bfly_plan_run_c2c(bfly_plan* plan, const float* in, float* out, uint32_t n, uint32_t batch) {
    PLAN_OR_FAIL();
    return p.run(in, out, n, batch);
}

int bfly_plan_run_c2c_many(bfly_plan* plan, const bfly_host_request* reqs, size_t count) {
    PLAN_OR_FAIL();
    if (!reqs || count == 0) return -8;
    std::vector<bfly::HostRequest> rs(count);
    for (size_t i = 0; i < count; ++i)
        rs[i] = {reqs[i].in, reqs[i].out, reqs[i].n, reqs[i].batch, reqs[i].direction, reqs[i].scale};
    return p.runMany(rs.data(), count);
}

int bfly_plan_run_r2c(bfly_plan* plan, const float* in, float* out, uint32_t n, uint32_t batch) {
    PLAN_OR_FAIL();
    return p.runR2C(in, out, n, batch);
}

int bfly_plan_run_c2r(bfly_plan* plan, const float* in, float* out, uint32_t n, uint32_t batch) {
    PLAN_OR_FAIL();
    return p.runC2R(in, out, n, batch);
}

int bfly_plan_measure(bfly_plan* plan, uint32_t n, uint32_t batch, bfly_metric* out) {
    PLAN_OR_FAIL();
    if (!out) return -1;
    bfly::Metric m;
    const int rc = p.measure(n, batch, &m);
    out->eta_us = m.etaUs;
    out->measured_us = m.measuredUs;
    out->max_rel_err = m.maxRelErr;
    out->measured_ok = m.measuredOk ? 1 : 0;
    return rc;
}

int bfly_plan_run_c2c_inverse(bfly_plan* plan, const float* in, float* out, uint32_t n,
                              uint32_t batch, float scale) {
    PLAN_OR_FAIL();
    return p.runInverse(in, out, n, batch, scale);
}

int bfly_plan_run_c2c_long(bfly_plan* plan, const float* in, float* out, uint32_t n, uint32_t batch,
                           int direction) {
    PLAN_OR_FAIL();
    return p.runLong(in, out, n, batch, direction);
}

int bfly_plan_exec_c2c_async(bfly_plan* plan, const void* d_in, void* d_out, uint32_t n,
                             uint64_t batch, int direction, float scale, void* stream) {
    PLAN_OR_FAIL();
    return p.execC2C(d_in, d_out, n, batch, direction, scale, stream);
}

int bfly_plan_exec_c2c_2d_async(bfly_plan* plan, const void* d_in, void* d_out, uint32_t ny,
                                uint32_t nx, uint64_t batch, int direction, float scale, void* stream) {
    PLAN_OR_FAIL();
    return p.execC2C2D(d_in, d_out, ny, nx, batch, direction, scale, stream);
}

int bfly_plan_exec_r2c_2d_async(bfly_plan* plan, const void* d_in, void* d_out, uint32_t ny,
                                uint32_t nx, uint64_t batch, float scale, void* stream) {
    PLAN_OR_FAIL();
    return p.execR2C2D(d_in, d_out, ny, nx, batch, scale, stream);
}

int bfly_plan_exec_c2r_2d_async(bfly_plan* plan, const void* d_in, void* d_out, uint32_t ny,
                                uint32_t nx, uint64_t batch, float scale, void* stream) {
    PLAN_OR_FAIL();
    return p.execC2R2D(d_in, d_out, ny, nx, batch, scale, stream);
}

int bfly_plan_exec_c2c_axis_async(bfly_plan* plan, const void* d_in, void* d_out, uint32_t n,
                                  uint64_t outer, uint64_t inner, int direction, float scale,
                                  void* stream) {
    PLAN_OR_FAIL();
    return p.execC2CAxis(d_in, d_out, n, outer, inner, direction, scale, stream);
}

int bfly_plan_exec_stft_async(bfly_plan* plan, const void* d_sig, void* d_out, uint32_t n,
                              uint64_t signals, uint64_t sig_len, uint32_t hop, int center,
                              const void* d_window, uint64_t* frames, void* stream) {
    PLAN_OR_FAIL();
    return p.execStft(d_sig, d_out, n, signals, sig_len, hop, center != 0, d_window, frames, stream);
}

int bfly_plan_exec_istft_async(bfly_plan* plan, const void* d_spec, void* d_out, uint32_t n,
                               uint64_t signals, uint32_t frames, uint32_t hop, int center,
                               const void* d_window, uint64_t out_len, float scale, void* stream) {
    PLAN_OR_FAIL();
    return p.execIstft(d_spec, d_out, n, signals, frames, hop, center != 0, d_window, out_len, scale, stream);
}

int bfly_plan_exec_stft_backward_async(bfly_plan* plan, const void* d_grad_spec, void* d_grad_sig, uint32_t n,
                                       uint64_t signals, uint64_t sig_len, uint32_t hop, int center,
                                       const void* d_window, void* stream) {
    PLAN_OR_FAIL();
    return p.execStftBackward(d_grad_spec, d_grad_sig, n, signals, sig_len, hop, center != 0, d_window, stream);
}

int bfly_plan_exec_istft_backward_async(bfly_plan* plan, const void* d_grad_out, void* d_grad_spec, uint32_t n,
                                        uint64_t signals, uint32_t frames, uint32_t hop, int center,
                                        const void* d_window, uint64_t out_len, float scale, void* stream) {
    PLAN_OR_FAIL();
    return p.execIstftBackward(d_grad_out, d_grad_spec, n, signals, frames, hop, center != 0, d_window, out_len,
                               scale, stream);
}

int bfly_plan_exec_r2c_async(bfly_plan* plan, const void* d_in, void* d_out, uint32_t n,
                             uint64_t batch, float s_edge, float s_int, void* stream) {
    PLAN_OR_FAIL();
    return p.execR2C(d_in, d_out, n, batch, s_edge, s_int, stream);
}

int bfly_plan_exec_c2r_async(bfly_plan* plan, const void* d_in, void* d_out, uint32_t n,
                             uint64_t batch, float s_edge, float s_int, float out_scale,
                             void* stream) {
    PLAN_OR_FAIL();
    return p.execC2R(d_in, d_out, n, batch, s_edge, s_int, out_scale, stream);
}

int bfly_plan_exec_c2c_tc_async(bfly_plan* plan, const void* d_in, void* d_out, uint32_t n,
                                uint64_t batch, int direction, float scale, int split_terms,
                                void* stream) {
    PLAN_OR_FAIL();
    return p.execC2CTensor(d_in, d_out, n, batch, direction, scale, split_terms, stream);
}

int bfly_tc_device_status(unsigned* status) { return bfly::Plan::tensorStatus(status); }
int bfly_long_device_status(unsigned* status) { return bfly::Plan::longStatus(status); }

static std::vector<bfly::RaggedRequest> raggedRequests(const bfly_ragged_request* reqs, size_t count) {
    std::vector<bfly::RaggedRequest> rs(count);
    for (size_t i = 0; i < count; ++i)
        rs[i] = {reqs[i].d_in, reqs[i].d_out, reqs[i].n, reqs[i].batch, reqs[i].direction, reqs[i].scale};
    return rs;
}

int bfly_ragged_create(bfly_plan* plan, const bfly_ragged_request* reqs, size_t count,
                       bfly_ragged** out) {
    if (!plan || !plan->plan || !out) return -10;
    *out = nullptr;
    if (!reqs || count == 0) return -8;
    const auto rs = raggedRequests(reqs, count);
    int status = 0;
    auto r = plan->plan->makeRagged(rs.data(), count, &status);
    if (!r) return status ? status : -1;
    *out = new bfly_ragged{std::move(r)};
    return 0;
}

int bfly_ragged_create_config(bfly_plan* plan, const bfly_ragged_request* reqs, size_t count, int mode,
                              uint32_t radix8, bfly_ragged** out) {
    if (!plan || !plan->plan || !out) return -10;
    *out = nullptr;
    if (!reqs || count == 0) return -8;
    const auto rs = raggedRequests(reqs, count);
    bfly::RaggedConfig cfg;
    cfg.mode = mode;
    cfg.radix8 = radix8;
    int status = 0;
    auto r = plan->plan->makeRagged(rs.data(), count, &status, &cfg);
    if (!r) return status ? status : -1;
    *out = new bfly_ragged{std::move(r)};
    return 0;
}

int bfly_context_tune_ragged(bfly_context* ctx, bfly_plan* plan, const bfly_ragged_request* reqs, size_t count,
                             bfly_ragged** out, char* log, size_t log_cap) {
    if (!ctx || !plan || !plan->plan || !out) return -10;
    *out = nullptr;
    if (!reqs || count == 0) return -8;
    const auto rs = raggedRequests(reqs, count);
    std::string text;
    int status = 0;
    auto r = ctx->ctx.tuneRagged(*plan->plan, rs.data(), count, &status, log ? &text : nullptr);
    if (log) copyOut(text, log, log_cap, nullptr);
    if (!r) return status ? status : -1;
    *out = new bfly_ragged{std::move(r)};
    return 0;
}

int bfly_ragged_config(bfly_ragged* ragged, int* mode, uint32_t* radix8) {
    if (!ragged || !ragged->ragged) return -10;
    const bfly::RaggedConfig c = ragged->ragged->config();
    if (mode) *mode = c.mode;
    if (radix8) *radix8 = c.radix8;
    return 0;
}

int bfly_ragged_exec_async(bfly_ragged* ragged, void* stream) {
    if (!ragged || !ragged->ragged) return -10;
    return ragged->ragged->exec(stream);
}

int bfly_ragged_info(bfly_ragged* ragged, uint64_t* tiles, int* grid, int* stages) {
    if (!ragged || !ragged->ragged) return -10;
    if (tiles) *tiles = ragged->ragged->tiles();
    if (grid) *grid = ragged->ragged->grid();
    if (stages) *stages = ragged->ragged->stages();
    return 0;
}

int bfly_ragged_device_status(unsigned* status) { return bfly::Ragged::deviceStatus(status); }

void bfly_ragged_destroy(bfly_ragged* ragged) { delete ragged; }

double bfly_max_rel_scaled(const float* got, const float* ref, size_t len) {
    return bfly::maxRelScaled(got, ref, len);
}
float bfly_pattern_at(size_t i) { return bfly::patternAt(i); }
uint32_t bfly_sample_batches(uint32_t batch, uint32_t want, uint32_t* out, uint32_t max_out) {
    return bfly::sampleBatches(batch, want, out, max_out);
}

}  // extern "C"
