// Host runtime of the batched FFT library: configuration loading, candidate enumeration,
// the measuring autotuner with a persisted choice cache, and the Plan entry points.
// Reference behaviour mirrored (TruNcat3/ascend-fft):
//   Hardware::load / DesignSpace::load   src/framework/butterfly.cpp:71-93, 326-350
//   enumerate / rank                     butterfly.cpp:383-512
//   Plan::prepare / run / runR2C / runC2R / measure   butterfly.cpp:587-924
//   Context::init / makePlan / select    butterfly.cpp:938-1102
// Status codes and the "guards before any allocation" rule follow the reference's
// docs/reference/api.md:34-50 and tests/test_runtime_guards.cpp:139-159.
// This file is plain C++: the GPU is reached only through backend.h.
#include "bfly/plan.hpp"

#include "backend.h"
#include "json_config.hpp"
#include "ragged.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <condition_variable>
#include <deque>
#include <functional>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <mutex>
#include <stdexcept>
#include <thread>
#include <utility>
#include <vector>

namespace bfly {

namespace {

constexpr uint32_t kMinN = 32;        // two passes of radix <= 16
constexpr uint32_t kMaxSinglePass = 16384;
constexpr uint32_t kMaxN = 65536;

// Ring slots of the "ring" schedule (k_long_ring.cu): BFLY_LONG_RING_MB megabytes, default 8.
size_t longRingSlotBytes() {
    const char* env = std::getenv("BFLY_LONG_RING_MB");
    const long mb = env ? std::strtol(env, nullptr, 10) : 8;
    return (size_t)(mb >= 1 && mb <= 1024 ? mb : 8) << 20;
}

std::string slurp(const std::string& path) {
    std::ifstream f(path, std::ios::binary);
    if (!f) throw std::runtime_error("cannot read configuration: " + path);
    return std::string(std::istreambuf_iterator<char>(f), std::istreambuf_iterator<char>());
}

bool pow2(uint64_t v) { return v && !(v & (v - 1)); }

int positiveInt(const json::Node& root, const char* key) {
    const long long v = root.get(key).asInt();
    if (v <= 0 || v > 0x7fffffffLL) throw std::runtime_error(std::string(key) + " must be a positive int");
    return (int)v;
}

const std::vector<json::Node>& axis(const json::Node& obj, const char* key) {
    const json::Node& v = obj.get(key);
    if (v.kind != json::Node::Array || v.items.empty())
        throw std::runtime_error(std::string(key) + " must be a nonempty array");
    return v.items;
}

void intAxis(const json::Node& obj, const char* key, std::vector<int>* out, int lo, int hi) {
    out->clear();
    for (const auto& v : axis(obj, key)) {
        const long long x = v.asInt();
        if (x < lo || x > hi) throw std::runtime_error(std::string(key) + " contains an invalid value");
        out->push_back((int)x);
    }
}

void stringAxis(const json::Node& obj, const char* key, std::vector<std::string>* out,
                std::initializer_list<const char*> allowed) {
    out->clear();
    for (const auto& v : axis(obj, key)) {
        const std::string& s = v.asString();
        bool ok = false;
        for (const char* a : allowed) ok = ok || s == a;
        if (!ok) throw std::runtime_error(std::string(key) + " contains unsupported value " + s);
        out->push_back(s);
    }
}

enum ShapeKind { kRunC2C, kRunR2C, kRunC2R, kRunLong, kPrepare, kMeasure, kExecC2C, kExecR2C, kExecC2R };

// Real transforms run an n/2-point complex FFT.
constexpr uint32_t kRealMin = 64, kRealMax = 8192;

}  // namespace

// ================================================================== H
Hardware Hardware::load(const std::string& path) {
    const json::Node root = json::parse(slurp(path));
    if (root.get("schema_version").asInt() != 1)
        throw std::runtime_error("unsupported hardware schema_version");
    Hardware hw;
    hw.gpu = root.get("gpu").asString();
    hw.arch = root.get("arch").asString();
    if (root.has("device_index")) {
        const long long d = root.get("device_index").asInt();
        if (d < 0 || d > 1024) throw std::runtime_error("device_index out of range");
        hw.deviceIndex = (int)d;
    }
    hw.smCount = positiveInt(root, "sm_count");
    hw.smemPerCta = positiveInt(root, "smem_bytes_per_cta");
    hw.smemPerSm = positiveInt(root, "smem_bytes_per_sm");
    hw.regsPerSm = positiveInt(root, "regs_per_sm");
    hw.maxThreadsPerSm = positiveInt(root, "max_threads_per_sm");
    if (root.has("l2_bytes")) {
        hw.l2Bytes = root.get("l2_bytes").asInt();
        if (hw.l2Bytes < 0) throw std::runtime_error("l2_bytes must be >= 0");
    }
    hw.hbmGbs = root.get("hbm_gbs").asDouble();
    if (!(hw.hbmGbs > 0.0) || hw.smemPerCta > hw.smemPerSm)
        throw std::runtime_error("hardware configuration contains nonpositive or inconsistent resources");
    return hw;
}

// ================================================================== A / P
bool Mapping::validate(const Hardware& hw, std::string* why) const {
    auto fail = [&](const char* m) {
        if (why) *why = m;
        return false;
    };
    if (ctaThreads <= 0) return fail("cta_threads must be > 0");
    if (ctaThreads > 1024 || ctaThreads % 32) return fail("cta_threads must be a multiple of 32 in [32, 1024]");
    if (hw.maxThreadsPerSm > 0 && ctaThreads > hw.maxThreadsPerSm) return fail("cta_threads exceeds max_threads_per_sm");
    if (level != 0) return fail("level!=0 (multi-GPU) is batch sharding above the plan, not a plan mapping");
    if (localExchange != "shared")
        return fail("local_exchange must be shared: the passes exchange through padded shared memory (a "
                    "16 x T register transpose by warp shuffles costs 64 SHFL + 128 SEL per thread against "
                    "32 shared-memory accesses)");
    return true;
}

size_t StagePlan::smemBytes(uint32_t n, int ctaThreads) const {
    if (radix <= 0 || n < (uint32_t)radix) return 0;
    const uint32_t T = n / (uint32_t)radix;
    if (!T || (uint32_t)ctaThreads < T) return 0;
    const uint32_t rows = (uint32_t)ctaThreads / T;
    uint32_t stride = (n - 1) + ((n - 1) >> 4) + 1;   // one pad word per 16
    if (T < 16) stride += ((T - stride % 16) % 16 + 16) % 16;
    return (size_t)rows * stride * 8u;
}

// ================================================================== space
DesignSpace DesignSpace::load(const std::string& path) {
    DesignSpace sp;
    sp.raw = slurp(path);
    const json::Node root = json::parse(sp.raw);
    if (root.get("schema_version").asInt() != 1)
        throw std::runtime_error("unsupported design-space schema_version");
    const json::Node& a = root.get("A");
    const json::Node& p = root.get("P");
    const json::Node& l = root.get("L");
    const json::Node& f = root.get("F");
    intAxis(a, "cta_threads", &sp.ctaThreads, 1, 1024);
    for (int c : sp.ctaThreads)
        if (c % 32) throw std::runtime_error("cta_threads must be multiples of 32");
    stringAxis(a, "local_exchange", &sp.localExchanges, {"shared"});
    intAxis(p, "radix", &sp.radices, 2, 16);
    for (int r : sp.radices)
        if (r != 2 && r != 4 && r != 8 && r != 16) throw std::runtime_error("radix must be 2, 4, 8 or 16");
    intAxis(p, "fusion_level", &sp.fusionStages, 1, 24);
    sp.coeffResidency.clear();
    for (const auto& v : axis(p, "coefficient_residency")) sp.coeffResidency.push_back(v.asBool() ? 1 : 0);
    stringAxis(l, "in", &sp.layoutsIn, {"interleaved", "planar"});
    stringAxis(l, "out", &sp.layoutsOut, {"interleaved", "planar"});
    stringAxis(f, "precision", &sp.precisions, {"fp32", "split_bf16"});
    stringAxis(f, "schedule", &sp.schedules, {"stockham", "four_step", "cluster", "ring"});
    return sp;
}

void DesignSpace::applyDefaults() {
    if (ctaThreads.empty()) ctaThreads = {128, 256, 512};
    if (radices.empty()) radices = {8, 16};
    if (fusionStages.empty()) fusionStages = {1};
    if (coeffResidency.empty()) coeffResidency = {1};
    if (localExchanges.empty()) localExchanges = {"shared"};
    if (layoutsIn.empty()) layoutsIn = {"interleaved"};
    if (layoutsOut.empty()) layoutsOut = {"interleaved"};
    if (precisions.empty()) precisions = {"fp32"};
    if (schedules.empty()) schedules = {"stockham", "four_step"};
}

const char* toString(State s) {
    switch (s) {
        case State::Infeasible: return "Infeasible";
        case State::Unverified: return "Unverified";
        case State::Feasible: return "Feasible";
        case State::Measured: return "Measured";
    }
    return "?";
}

// ================================================================== estimate
// Roofline estimate: compulsory HBM bytes at the profile's measured bandwidth, a fixed launch
// cost, a per-extra-pass smem term, and a second HBM round trip for the four-step schedule.
Metric estimate(const Hardware& hw, const Candidate& c, uint32_t n, uint32_t batch) {
    Metric m;
    if (!n || !batch || hw.hbmGbs <= 0) return m;
    const double bytes = 16.0 * (double)n * (double)batch;
    const double hbmUs = bytes / (hw.hbmGbs * 1e3);
    int logn = 0;
    while ((1u << logn) < n) ++logn;
    int loge = 0;
    while (c.p.radix > 1 && (1 << loge) < c.p.radix) ++loge;
    const int passes = loge ? (logn + loge - 1) / loge : logn;
    double us = 2.5 + hbmUs * (1.0 + 0.04 * std::max(0, passes - 2));
    if (c.f.schedule == "four_step") us = 3.0 + 2.0 * hbmUs;
    if (c.f.schedule == "cluster") us = 3.0 + 1.3 * hbmUs;
    if (c.f.schedule == "ring") us = 3.0 + 2.4 * hbmUs;   // measured 0.84-0.97x of four_step
    if (c.a.ctaThreads < 256) us *= 1.02;
    m.etaUs = us;
    return m;
}

// ================================================================== enumerate
std::vector<Candidate> enumerate(const DesignSpace& sp, const Hardware& hw, uint32_t n,
                                 uint32_t batch) {
    std::vector<Candidate> out;
    auto pack = [](const std::string& s) { return s == "planar" ? Layout::Planar : Layout::Interleaved; };
    char buf[256];
    for (int cta : sp.ctaThreads)
      for (int radix : sp.radices)
        for (int fl : sp.fusionStages)
          for (int cr : sp.coeffResidency)
            for (const std::string& lx : sp.localExchanges)
              for (const std::string& li : sp.layoutsIn)
                for (const std::string& lo : sp.layoutsOut)
                  for (const std::string& prec : sp.precisions)
                    for (const std::string& sched : sp.schedules) {
        Candidate c;
        c.a.ctaThreads = cta;
        c.a.localExchange = lx;
        c.p.radix = radix;
        c.p.fusionLevel = fl;
        c.p.coefficientResidency = cr != 0;
        c.l.in = pack(li);
        c.l.out = pack(lo);
        c.f.precision = prec;
        c.f.schedule = sched;
        std::snprintf(buf, sizeof(buf), "r%d_cta%d_%s_%s_%s", radix, cta, lx.c_str(), prec.c_str(), sched.c_str());
        c.id = buf;
        if (fl != 1) c.id += "_f" + std::to_string(fl);
        if (c.l.in == Layout::Planar) c.id += "_inplanar";
        if (c.l.out == Layout::Planar) c.id += "_outplanar";
        if (!c.p.coefficientResidency) c.id += "_noRes";

        auto infeasible = [&](const std::string& why) {
            c.state = State::Infeasible;
            c.reason = why;
        };
        std::string why;
        const uint32_t T = radix > 0 ? n / (uint32_t)radix : 0;
        if (!c.a.validate(hw, &why)) {
            infeasible(why);
        } else if (!c.p.coefficientResidency) {
            infeasible("kernels read twiddle tables through L1; coefficient_residency=false is not lowered");
        } else if (!pow2(n)) {
            infeasible("n must be a power of two");
        } else if (n < kMinN) {
            infeasible("n below the 32-point minimum (two passes of radix <= 16)");
        } else if (n > kMaxN) {
            infeasible("n exceeds the 65536-point envelope");
        } else if (batch == 0) {
            infeasible("batch must be positive");
        } else if ((uint64_t)batch * 2ull * n > 0xFFFFFFFFull) {
            std::snprintf(buf, sizeof(buf),
                          "batch*2*n = %llu exceeds the uint32 element offsets of the host-pointer API "
                          "(max batch for n=%u is %llu)",
                          (unsigned long long)batch * 2ull * n, n,
                          (unsigned long long)(0xFFFFFFFFull / (2ull * n)));
            infeasible(buf);
        } else if (c.l.in != Layout::Interleaved || c.l.out != Layout::Interleaved) {
            infeasible("planar layout is not lowered (kernels consume and produce interleaved fp32)");
        } else if (fl != 1) {
            infeasible("fusion_level!=1 is not lowered (each schedule fuses all of its passes)");
        } else if (prec != "fp32") {
            infeasible("split_bf16 is served by the tensor-core entry points, not by plan candidates");
        } else if (sched == "cluster") {
            if (n < 8192) infeasible("cluster schedule is only used for n >= 8192");
            else if (radix != 16) infeasible("cluster kernels use radix 16");
            else if (!backend::hasLongCluster(n, cta))
                infeasible("no cluster kernel for this (n, cta_threads): 256 threads per CTA, or 512 for n >= 16384");
            else c.state = State::Unverified;
        } else if (sched == "ring") {
            if (!backend::hasLongRing(n)) infeasible("ring schedule serves n = 8192 .. 65536");
            else if (radix != backend::longE() || cta != 256)
                infeasible("ring kernels use radix 16 and 256-thread CTAs");
            else c.state = State::Unverified;
        } else if (sched == "four_step") {
            uint32_t n1 = 0, n2 = 0;
            backend::longSplit(n, &n1, &n2);
            if (n <= 4096) infeasible("four_step is only used for n > 4096");
            else if (!n1 || !backend::hasLongSplit(n1, n2)) infeasible("no four-step split for this n");
            else if (radix != backend::longE() || cta != 256)
                infeasible("four_step kernels use radix 16 and 256-thread CTAs");
            else c.state = State::Unverified;
        } else {   // stockham single pass
            const size_t smem = c.p.smemBytes(n, cta);
            if (n > kMaxSinglePass) {
                infeasible("single-pass stockham holds at most 16384 points in shared memory");
            } else if ((uint32_t)radix > n / 2) {
                infeasible("radix must leave at least two passes (radix <= n/2)");
            } else if (T > (uint32_t)cta || (uint32_t)cta % T) {
                std::snprintf(buf, sizeof(buf), "n/radix = %u threads per transform do not tile cta_threads=%d", T, cta);
                infeasible(buf);
            } else if (smem > (size_t)hw.smemPerCta) {
                std::snprintf(buf, sizeof(buf), "shared memory %.1f KiB > %d KiB per CTA (radix=%d, n=%u)",
                              smem / 1024.0, hw.smemPerCta / 1024, radix, n);
                infeasible(buf);
            } else if (!backend::hasVariant(backend::kC2C, n, radix, cta)) {
                std::snprintf(buf, sizeof(buf), "no compiled kernel for (n=%u, radix=%d, cta=%d)", n, radix, cta);
                infeasible(buf);
            } else {
                c.state = State::Unverified;
            }
        }
        c.q = estimate(hw, c, n, batch);
        out.push_back(std::move(c));
    }
    return out;
}

std::vector<const Candidate*> rank(const std::vector<Candidate>& cs) {
    std::vector<const Candidate*> v;
    for (const auto& c : cs)
        if (c.state != State::Infeasible) v.push_back(&c);
    std::stable_sort(v.begin(), v.end(), [](const Candidate* x, const Candidate* y) {
        if (x->state != y->state) return x->state > y->state;
        return x->q.etaUs < y->q.etaUs;
    });
    return v;
}

// A candidate the kernels can execute (independent of n).
static bool lowerable(const Candidate& c, const Hardware& hw) {
    return c.a.validate(hw, nullptr) && c.p.coefficientResidency && c.p.fusionLevel == 1 &&
           (c.p.radix == 8 || c.p.radix == 16) && c.l.contiguous &&
           c.l.in == Layout::Interleaved && c.l.out == Layout::Interleaved &&
           c.f.precision == "fp32" &&
           (c.f.schedule == "stockham" || c.f.schedule == "four_step" || c.f.schedule == "cluster" ||
            c.f.schedule == "ring") &&
           (c.a.ctaThreads == 128 || c.a.ctaThreads == 256 || c.a.ctaThreads == 512 ||
            c.a.ctaThreads == 1024);
}

// ================================================================== Plan
struct Plan::Impl {
    Hardware hw;
    int device = 0;
    std::map<std::pair<uint32_t, int>, void*> twC2C;   // (n, e) -> Stockham table
    std::map<uint32_t, void*> twReal;                  // n -> W_n^k, k <= n/2
    struct LongTw {
        void* lo = nullptr;
        void* hi = nullptr;
    };
    std::map<uint32_t, LongTw> twLong;                 // n -> two-level W_n tables
    void* devIn = nullptr;
    void* devOut = nullptr;
    void* devWork = nullptr;
    size_t devInCap = 0, devOutCap = 0, devWorkCap = 0;
    void* devRingCtr = nullptr;   // item counters of the L2-ring long C2C
    size_t devRingCtrCap = 0;
    backend::Timer* timer = nullptr;
    void* aux[2] = {nullptr, nullptr};   // upload / download streams of the pipelined host round trip
    void* ev[2] = {nullptr, nullptr};    // chunk uploaded / chunk transformed
    void* devHalf = nullptr;             // column-transformed half spectrum of execC2R2D
    size_t devHalfCap = 0;
    // pinned staging for pageable host buffers: two slots per direction, with the events that
    // say a slot's upload has read it / its download has filled it
    void* pinIn[2] = {nullptr, nullptr};
    void* pinOut[2] = {nullptr, nullptr};
    size_t pinInCap = 0, pinOutCap = 0;
    void* evStage[2] = {nullptr, nullptr};
    void* evOut[2] = {nullptr, nullptr};
    void* tcTable[4] = {nullptr, nullptr, nullptr, nullptr};   // split DFT-16 operand per term count
    std::map<uint32_t, void*> twTc;                            // n -> tensor-core pass twiddles by row
    struct Chirp {
        void* chirp = nullptr;   // c[j] = exp(-i*pi*j^2/n), j < n
        void* filt = nullptr;    // FFT_M of the padded conj(c) sequence, / M
    };
    std::map<uint32_t, Chirp> bluestein;   // non-power-of-two n -> Bluestein tables
    std::map<uint32_t, void*> dftSmall;    // A -> W_A^m, m < A (prime-factor kernels)
    struct Mixed {
        backend::MixedRadix plan;   // passes of the mixed-radix kernel
        void* tw = nullptr;         // their twiddles (plan.twsize entries)
    };
    std::map<uint32_t, Mixed> mixed;   // 7-smooth n served by the mixed-radix kernel
};

Plan::Plan(Candidate c) : cand_(std::move(c)) {}

Plan::~Plan() {
    if (!impl_) return;
    for (auto& kv : impl_->twC2C) if (kv.second) backend::release(kv.second);
    for (auto& kv : impl_->twReal) if (kv.second) backend::release(kv.second);
    for (auto& kv : impl_->twLong) {
        if (kv.second.lo) backend::release(kv.second.lo);
        if (kv.second.hi) backend::release(kv.second.hi);
    }
    if (impl_->devIn) backend::release(impl_->devIn);
    if (impl_->devOut) backend::release(impl_->devOut);
    if (impl_->devWork) backend::release(impl_->devWork);
    if (impl_->devRingCtr) backend::release(impl_->devRingCtr);
    if (impl_->devHalf) backend::release(impl_->devHalf);
    for (int i = 0; i < 2; ++i) {
        if (impl_->pinIn[i]) backend::releaseHost(impl_->pinIn[i]);
        if (impl_->pinOut[i]) backend::releaseHost(impl_->pinOut[i]);
        if (impl_->evStage[i]) backend::eventDestroy(impl_->evStage[i]);
        if (impl_->evOut[i]) backend::eventDestroy(impl_->evOut[i]);
    }
    backend::timerDestroy(impl_->timer);
    for (void* st : impl_->aux)
        if (st) backend::streamDestroy(st);
    for (void* e : impl_->ev)
        if (e) backend::eventDestroy(e);
    for (auto& kv : impl_->twTc)
        if (kv.second) backend::release(kv.second);
    for (void* t : impl_->tcTable)
        if (t) backend::release(t);
    for (auto& kv : impl_->dftSmall)
        if (kv.second) backend::release(kv.second);
    for (auto& kv : impl_->mixed)
        if (kv.second.tw) backend::release(kv.second.tw);
    for (auto& kv : impl_->bluestein) {
        if (kv.second.chirp) backend::release(kv.second.chirp);
        if (kv.second.filt) backend::release(kv.second.filt);
    }
}

static int ensureBuf(void** p, size_t* cap, size_t bytes) {
    if (*cap >= bytes && *p) return 0;
    if (*p) {
        backend::release(*p);
        *p = nullptr;
    }
    *cap = 0;
    if (backend::alloc(p, bytes)) {
        *p = nullptr;
        return -1;
    }
    *cap = bytes;
    return 0;
}

// Real transforms of even n whose half length runs the mixed-radix kernel.
static bool realMixed(uint32_t n) { return n >= 4 && n % 2 == 0 && backend::mixedRadix(n / 2, nullptr); }

bool Plan::validShape(uint32_t n, uint32_t batch, int kind) const {
    if (!impl_ || batch == 0) return false;
    // lengths outside the power-of-two kernels (non-powers of two, and 2..16) only through the
    // device-pointer entries: C2C by the prime-factor kernel for A*2^k, mixed radix for other
    // 13-smooth lengths, else Bluestein; R2C / C2R of even n with n/2 13-smooth by mixed radix
    if (!pow2(n) || (kind == kExecC2C && n < kMinN)) {
        uint32_t a = 0, b = 0;
        if (kind == kExecR2C || kind == kExecC2R) return realMixed(n);
        return kind == kExecC2C &&
               (backend::bluesteinM(n) != 0 || backend::pfaSplit(n, &a, &b) || backend::mixedRadix(n, nullptr));
    }
    const bool offsetGuard = kind == kRunC2C || kind == kRunR2C || kind == kRunC2R ||
                             kind == kRunLong || kind == kMeasure;
    switch (kind) {
        case kRunC2C: if (n < 64 || n > 4096) return false; break;
        case kRunR2C: if (n < 128 || n > 8192) return false; break;
        case kRunC2R: if (n < 64 || n > 4096) return false; break;
        case kRunLong: if (n < 8192 || n > kMaxN) return false; break;
        case kPrepare:
        case kMeasure:
        case kExecC2C: if (n < kMinN || n > kMaxN) return false; break;
        case kExecR2C:
        case kExecC2R: if (n < kRealMin || n > kRealMax) return false; break;
        default: return false;
    }
    if (offsetGuard && (uint64_t)batch * 2ull * n > 0xFFFFFFFFull) return false;
    int e = 0, cta = 0;
    const int rk = (kind == kRunR2C || kind == kExecR2C) ? backend::kR2C
                 : (kind == kRunC2R || kind == kExecC2R) ? backend::kC2R : backend::kC2C;
    return resolve(rk, n, &e, &cta) == 0;
}

// Kernel variant for (kind, n): the candidate's radix/cta when compiled for n (one CTA per
// transform, e = radix); otherwise, for long C2C lengths, the four-step kernels (e = 0), or one
// thread-block cluster per row (e = -1) when the candidate is scheduled "cluster".  Measured on
// B200 at batch*n = 2^26 the two-kernel four-step is the faster of the two at every long n
// (the cluster kernel is bound by instruction issue at 16 resident warps per SM), so it is
// the default.
int Plan::resolve(int kind, uint32_t n, int* e, int* cta) const {
    const int r = cand_.p.radix, c = cand_.a.ctaThreads;
    if (kind == backend::kC2C) {
        const std::string& sched = cand_.f.schedule;
        if (sched == "stockham" && n <= kMaxSinglePass && backend::hasVariant(backend::kC2C, n, r, c)) {
            *e = r;
            *cta = c;
            return 0;
        }
        if (sched == "ring" && backend::hasLongRing(n)) {
            *e = -2;
            *cta = 256;
            return 0;
        }
        if (sched == "cluster" && backend::hasLongCluster(n, 256)) {
            *e = -1;
            *cta = backend::hasLongCluster(n, c) ? c : 256;
            return 0;
        }
        uint32_t n1 = 0, n2 = 0;
        backend::longSplit(n, &n1, &n2);
        if (n1 && backend::hasLongSplit(n1, n2)) {
            *e = 0;
            *cta = 256;
            return 0;
        }
        return -1;
    }
    if (!backend::hasVariant(kind, n, r, c)) return -1;
    *e = r;
    *cta = c;
    return 0;
}

int Plan::prepareC2C(uint32_t n, int e) {
    const auto key = std::make_pair(n, e);
    if (impl_->twC2C.count(key)) return 0;
    const size_t count = backend::stockhamTwiddleCount(n, e);
    void* tw = nullptr;
    if (count) {
        if (backend::alloc(&tw, count * 8)) return -1;
        if (backend::buildStockhamTwiddles(tw, n, e, stream_) || backend::streamSync(stream_)) {
            backend::release(tw);
            return -1;
        }
    }
    impl_->twC2C[key] = tw;
    return 0;
}

int Plan::prepareReal(uint32_t n) {
    if (impl_->twReal.count(n)) return 0;
    void* tw = nullptr;
    const int count = (int)(n / 2 + 1);
    if (backend::alloc(&tw, (size_t)count * 8)) return -1;
    if (backend::buildLinearTwiddles(tw, count, 1, n, stream_) || backend::streamSync(stream_)) {
        backend::release(tw);
        return -1;
    }
    impl_->twReal[n] = tw;
    return 0;
}

int Plan::prepareLong(uint32_t n) {
    uint32_t n1 = 0, n2 = 0;
    backend::longSplit(n, &n1, &n2);
    if (!n1) return -1;
    if (prepareC2C(n1, backend::longE()) || prepareC2C(n2, backend::longE())) return -1;
    if (impl_->twLong.count(n)) return 0;
    Impl::LongTw t;
    const int nhi = (int)(n / 256);
    if (backend::alloc(&t.lo, 256 * 8)) return -1;
    if (backend::alloc(&t.hi, (size_t)nhi * 8)) {
        backend::release(t.lo);
        return -1;
    }
    if (backend::buildLinearTwiddles(t.lo, 256, 1, n, stream_) ||
        backend::buildLinearTwiddles(t.hi, nhi, 256, n, stream_) || backend::streamSync(stream_)) {
        backend::release(t.lo);
        backend::release(t.hi);
        return -1;
    }
    impl_->twLong[n] = t;
    return 0;
}

int Plan::preparePfa(uint32_t n) {
    uint32_t a = 0, b = 0;
    if (!backend::pfaSplit(n, &a, &b) || prepareC2C(b, kColsE)) return -1;
    if (impl_->dftSmall.count(a)) return 0;
    void* w = nullptr;
    if (backend::alloc(&w, (size_t)a * 8)) return -1;
    if (backend::buildLinearTwiddles(w, (int)a, 1, a, stream_) || backend::streamSync(stream_)) {
        backend::release(w);
        return -1;
    }
    impl_->dftSmall[a] = w;
    return 0;
}

int Plan::prepareMixed(uint32_t n) {
    if (impl_->mixed.count(n)) return 0;
    Impl::Mixed m;
    if (!backend::mixedRadix(n, &m.plan)) return -1;
    if (backend::alloc(&m.tw, (size_t)std::max(m.plan.twsize, 1) * 8)) return -1;
    if (backend::buildMixedTwiddles(m.tw, m.plan, stream_) || backend::streamSync(stream_)) {
        backend::release(m.tw);
        return -1;
    }
    impl_->mixed[n] = m;
    return 0;
}

int Plan::prepareAnyLength(uint32_t n) {
    uint32_t a = 0, b = 0;
    if (!pow2(n) && backend::pfaSplit(n, &a, &b)) return preparePfa(n);
    if (backend::mixedRadix(n, nullptr)) return prepareMixed(n);
    return prepareBluestein(n);
}

int Plan::prepareBluestein(uint32_t n) {
    const uint32_t M = backend::bluesteinM(n);
    if (!M || prepareC2C(M, kColsE)) return -1;
    if (impl_->bluestein.count(n)) return 0;
    Impl::Chirp t;
    void* scratch = nullptr;
    if (backend::alloc(&t.chirp, (size_t)n * 8) || backend::alloc(&t.filt, (size_t)M * 8) ||
        backend::alloc(&scratch, (size_t)M * 16)) {
        if (t.chirp) backend::release(t.chirp);
        if (t.filt) backend::release(t.filt);
        return -1;
    }
    const bool bad = backend::buildBluesteinTables(t.chirp, t.filt, scratch, n, stream_) ||
                     backend::streamSync(stream_);
    backend::release(scratch);
    if (bad) {
        backend::release(t.chirp);
        backend::release(t.filt);
        return -1;
    }
    impl_->bluestein[n] = t;
    return 0;
}

int Plan::prepare(uint32_t n, uint32_t batch) {
    if (!validShape(n, batch, kPrepare)) return -8;
    int e = 0, cta = 0;
    if (resolve(backend::kC2C, n, &e, &cta)) return -8;
    const int rcode = e > 0 ? prepareC2C(n, e) : prepareLong(n);
    if (rcode) return -1;
    tf_.clear();
    tf_.push_back({Transform::GenTwiddles, "FP64 twiddle tables built on the device, rounded to fp32"});
    tf_.push_back({Transform::LaunchKernel, e > 0 ? "stockham single-pass kernel on the context stream"
                                            : e == -1 ? "one thread-block cluster per row (on-chip transpose)"
                                            : e == -2 ? "one persistent four-step launch, intermediate in an L2 ring"
                                                      : "four-step column + row kernels on the context stream"});
    return 0;
}

int Plan::execC2C(const void* dIn, void* dOut, uint32_t n, uint64_t batch, int direction,
                  float scale, void* stream) {
    return execC2CWith(dIn, dOut, n, batch, direction, scale, stream, nullptr);
}

// `work`: four-step workspace of n*batch complex values, or nullptr for the plan-owned one.
int Plan::execC2CWith(const void* dIn, void* dOut, uint32_t n, uint64_t batch, int direction,
                      float scale, void* stream, void* work) {
    if (!dIn || !dOut || batch == 0 || batch > 0xFFFFFFFFull || (direction != -1 && direction != 1))
        return -8;
    if (!validShape(n, (uint32_t)batch, kExecC2C)) return -8;
    void* s = stream;   // NULL is the CUDA default stream
    const bool inv = direction > 0;
    uint32_t pa = 0, pb = 0;
    if (!pow2(n) && backend::pfaSplit(n, &pa, &pb)) {   // n = A * 2^k: prime-factor kernel
        if (preparePfa(n)) return -2;
        if (backend::launchPfa(dIn, dOut, n, batch, inv, scale, impl_->twC2C[{pb, kColsE}], impl_->dftSmall[pa], s))
            return -5;
        return 0;
    }
    if ((!pow2(n) || n < kMinN) && backend::mixedRadix(n, nullptr)) {   // other 7-smooth lengths
        if (prepareMixed(n)) return -2;
        const auto& m = impl_->mixed[n];
        if (backend::launchMixed(dIn, dOut, m.plan, batch, inv, scale, m.tw, s)) return -5;
        return 0;
    }
    if (!pow2(n) || n < kMinN) {   // Bluestein: one kernel on the padded power-of-two length
        if (prepareBluestein(n)) return -2;
        const auto& t = impl_->bluestein[n];
        if (backend::launchBluestein(dIn, dOut, n, batch, inv, scale,
                                     impl_->twC2C[{backend::bluesteinM(n), kColsE}], t.chirp, t.filt, s))
            return -5;
        return 0;
    }
    int e = 0, cta = 0;
    if (resolve(backend::kC2C, n, &e, &cta)) return -1;
    if (e > 0) {
        if (prepareC2C(n, e)) return -2;
        if (backend::launchC2C(dIn, dOut, n, batch, inv, scale, impl_->twC2C[{n, e}], e, cta, s)) return -5;
        return 0;
    }
    if (prepareLong(n)) return -2;
    uint32_t n1 = 0, n2 = 0;
    backend::longSplit(n, &n1, &n2);
    if (e == -1) {
        const auto& lt = impl_->twLong[n];
        const int E = backend::longE();
        const int rc = backend::launchLongCluster(dIn, dOut, n, batch, inv, scale, impl_->twC2C[{n1, E}],
                                                  impl_->twC2C[{n2, E}], lt.lo, lt.hi, cta, s);
        if (rc == 0) return 0;
        if (rc != backend::kLongClusterUnaligned) return -5;
        // an input the tensor map cannot address: the four-step kernels below take any float2 pointer
    }
    const auto& lt = impl_->twLong[n];
    const int E = backend::longE();
    if (e == -2 && !work) {
        // one persistent launch, the intermediate in an L2-resident ring of three row slots
        const uint32_t slotRows = backend::longRingSlotRows(n, batch, longRingSlotBytes());
        const uint64_t chunks = (batch + slotRows - 1) / slotRows;
        const size_t ringBytes = (size_t)std::min<uint64_t>(chunks, (uint64_t)backend::longRingSlots()) * slotRows * n * 8;
        if (ensureBuf(&impl_->devWork, &impl_->devWorkCap, ringBytes) ||
            ensureBuf(&impl_->devRingCtr, &impl_->devRingCtrCap, 64))
            return -3;
        if (backend::launchLongRing(dIn, dOut, impl_->devWork, slotRows, n, batch, inv, scale,
                                    impl_->twC2C[{n1, E}], impl_->twC2C[{n2, E}], lt.lo, lt.hi,
                                    impl_->devRingCtr, s))
            return -5;
        return 0;
    }
    if (!work) {
        if (ensureBuf(&impl_->devWork, &impl_->devWorkCap, (size_t)n * batch * 8)) return -3;
        work = impl_->devWork;
    }
    if (backend::launchLongA(dIn, work, n1, n2, batch, inv, impl_->twC2C[{n1, E}], lt.lo, lt.hi, s))
        return -5;
    if (backend::launchLongB(work, dOut, n1, n2, batch, inv, scale, impl_->twC2C[{n2, E}], s))
        return -5;
    return 0;
}

int Plan::execC2CTensor(const void* dIn, void* dOut, uint32_t n, uint64_t batch, int direction,
                        float scale, int splitTerms, void* stream) {
    if (!impl_ || !dIn || !dOut || batch == 0 || batch > 0xFFFFFFFFull ||
        (direction != -1 && direction != 1) || !backend::hasTensorVariant(n, splitTerms))
        return -8;
    if (prepareC2C(n, 16)) return -2;
    void*& table = impl_->tcTable[splitTerms];
    if (!table) {
        void* t = nullptr;
        if (backend::alloc(&t, backend::tensorTableBytes(splitTerms))) return -3;
        if (backend::buildTensorTable(t, splitTerms, stream_) || backend::streamSync(stream_)) {
            backend::release(t);
            return -2;
        }
        table = t;
    }
    if (!impl_->twTc.count(n)) {
        void* t = nullptr;
        const size_t count = backend::tensorTwiddleCount(n);
        if (count) {
            if (backend::alloc(&t, count * 8)) return -3;
            if (backend::buildTensorTwiddles(t, n, stream_) || backend::streamSync(stream_)) {
                backend::release(t);
                return -2;
            }
        }
        impl_->twTc[n] = t;
    }
    if (backend::launchC2CTensor(dIn, dOut, n, batch, direction > 0, scale, impl_->twC2C[{n, 16}],
                                 impl_->twTc[n], table, splitTerms, stream))
        return -5;
    return 0;
}

int Plan::tensorStatus(unsigned* status) {
    if (!status) return -10;
    return backend::tensorStatus(status, true) ? -6 : 0;
}

int Plan::longStatus(unsigned* status) {
    if (!status) return -10;
    unsigned ring = 0;
    if (backend::longClusterStatus(status, true) || backend::longRingStatus(&ring, true)) return -6;
    *status |= ring ? 2u : 0u;
    return 0;
}

// Column pass shared by the 2-D and axis entry points: n-point transforms down `cols`
// columns of `mats` matrices with row pitch `pitch`.
int Plan::execCols(const void* dIn, void* dOut, uint32_t n, uint64_t mats, uint32_t cols,
                   uint64_t pitch, bool inverse, float scale, void* stream) {
    if (!backend::hasCols(n)) return -8;
    if (prepareC2C(n, kColsE)) return -2;
    if (backend::launchCols(dIn, dOut, n, cols, pitch, (uint64_t)n * pitch, mats, inverse, scale,
                            impl_->twC2C[{n, kColsE}], stream))
        return -5;
    return 0;
}

int Plan::execC2C2D(const void* dIn, void* dOut, uint32_t ny, uint32_t nx, uint64_t batch,
                    int direction, float scale, void* stream) {
    if (!dIn || !dOut || batch == 0 || (direction != -1 && direction != 1)) return -8;
    if (!pow2(ny) || !backend::hasCols(ny)) return -8;
    if (batch > 0xFFFFFFFFull / ny || !validShape(nx, (uint32_t)(batch * ny), kExecC2C)) return -8;
    if (int r = execC2CWith(dIn, dOut, nx, batch * ny, direction, 1.0f, stream, nullptr)) return r;
    return execCols(dOut, dOut, ny, batch, nx, nx, direction > 0, scale, stream);
}

int Plan::execC2CAxis(const void* dIn, void* dOut, uint32_t n, uint64_t outer, uint64_t inner,
                      int direction, float scale, void* stream) {
    if (!dIn || !dOut || outer == 0 || inner == 0 || (direction != -1 && direction != 1)) return -8;
    if (inner == 1) return execC2C(dIn, dOut, n, outer, direction, scale, stream);
    if (!pow2(n) || !backend::hasCols(n) || inner > 0xFFFFFFFFull) return -8;
    if (outer > (~0ull) / n / inner) return -8;
    return execCols(dIn, dOut, n, outer, (uint32_t)inner, inner, direction > 0, scale, stream);
}

int Plan::execStft(const void* dSig, void* dOut, uint32_t n, uint64_t signals, uint64_t sigLen,
                   uint32_t hop, bool center, const void* dWindow, uint64_t* framesOut, void* stream) {
    const bool mixedN = !pow2(n) && realMixed(n);
    if (!impl_ || !dSig || !dOut || signals == 0 || hop == 0 || !(backend::hasStft(n) || mixedN)) return -8;
    if (reinterpret_cast<uintptr_t>(dWindow) & 7u) return -8;   // the kernels read the window as float2
    if (center ? sigLen <= n / 2 : sigLen < n) return -8;
    const uint64_t frames = center ? 1 + sigLen / hop : 1 + (sigLen - n) / hop;
    if (frames > 0xFFFFFFFFull || signals > (~0ull) / frames) return -8;
    if (framesOut) *framesOut = frames;
    if (mixedN) {
        if (prepareMixed(n / 2) || prepareReal(n)) return -2;
        const auto& m = impl_->mixed[n / 2];
        if (backend::launchStftMixed(dSig, dOut, m.plan, signals, (uint32_t)frames, sigLen, sigLen, hop, center,
                                     dWindow, m.tw, impl_->twReal[n], stream))
            return -5;
        return 0;
    }
    if (prepareC2C(n / 2, kColsE) || prepareReal(n)) return -2;
    if (backend::launchStft(dSig, dOut, n, signals, (uint32_t)frames, sigLen, sigLen, hop, center, dWindow,
                            impl_->twC2C[{n / 2, kColsE}], impl_->twReal[n], stream))
        return -5;
    return 0;
}

int Plan::execStftBackward(const void* dGradSpec, void* dGradSig, uint32_t n, uint64_t signals, uint64_t sigLen,
                           uint32_t hop, bool center, const void* dWindow, void* stream) {
    if (!impl_ || !dGradSpec || !dGradSig || signals == 0 || hop == 0 || hop > n || !backend::hasStft(n)) return -8;
    if (reinterpret_cast<uintptr_t>(dWindow) & 7u) return -8;
    if (center ? sigLen < (uint64_t)n + 2 : sigLen < n) return -8;
    const uint64_t frames = center ? 1 + sigLen / hop : 1 + (sigLen - n) / hop;
    if (frames > 0xFFFFFFFFull || signals > 0xFFFFFFFFull / frames) return -8;
    if (prepareC2C(n / 2, kColsE) || prepareReal(n)) return -2;
    if (backend::launchStftAdjoint(dGradSpec, dGradSig, n, signals, (uint32_t)frames, hop, center, sigLen, dWindow,
                                   impl_->twC2C[{n / 2, kColsE}], impl_->twReal[n], stream))
        return -5;
    return 0;
}

int Plan::execIstftBackward(const void* dGradOut, void* dGradSpec, uint32_t n, uint64_t signals, uint32_t frames,
                            uint32_t hop, bool center, const void* dWindow, uint64_t outLen, float scale,
                            void* stream) {
    if (!impl_ || !dGradOut || !dGradSpec || signals == 0 || frames == 0 || hop == 0 || hop > n ||
        !backend::hasStft(n))
        return -8;
    if (signals > 0xFFFFFFFFull / frames || outLen == 0 || outLen > (1ull << 62)) return -8;
    if (reinterpret_cast<uintptr_t>(dWindow) & 7u) return -8;
    if (prepareC2C(n / 2, kColsE) || prepareReal(n)) return -2;
    if (backend::launchIstftAdjoint(dGradOut, dGradSpec, n, signals, frames, hop, center ? (int64_t)(n / 2) : 0,
                                    outLen, dWindow, impl_->twC2C[{n / 2, kColsE}], impl_->twReal[n], scale, stream))
        return -5;
    return 0;
}

int Plan::execIstft(const void* dSpec, void* dOut, uint32_t n, uint64_t signals, uint32_t frames, uint32_t hop,
                    bool center, const void* dWindow, uint64_t outLen, float scale, void* stream) {
    const bool mixedN = !pow2(n) && realMixed(n) && n <= backend::kIstftMixedMaxN;
    if (!impl_ || !dSpec || !dOut || signals == 0 || frames == 0 || hop == 0 || hop > n ||
        !(backend::hasStft(n) || mixedN))
        return -8;
    if (signals > 0xFFFFFFFFull / frames || outLen == 0 || outLen > (1ull << 62)) return -8;
    if (reinterpret_cast<uintptr_t>(dWindow) & 7u) return -8;   // the kernels read the window as float2
    if (mixedN) {
        if (prepareMixed(n / 2) || prepareReal(n)) return -2;
        const auto& m = impl_->mixed[n / 2];
        if (backend::launchIstftMixed(dSpec, dOut, m.plan, signals, frames, hop, center ? (int64_t)(n / 2) : 0, outLen,
                                      dWindow, m.tw, impl_->twReal[n], scale, stream))
            return -5;
        return 0;
    }
    if (prepareC2C(n / 2, kColsE) || prepareReal(n)) return -2;
    if (backend::launchIstft(dSpec, dOut, n, signals, frames, hop, center ? (int64_t)(n / 2) : 0, outLen, dWindow,
                             impl_->twC2C[{n / 2, kColsE}], impl_->twReal[n], scale, stream))
        return -5;
    return 0;
}

int Plan::execR2C(const void* dIn, void* dOut, uint32_t n, uint64_t batch, float sEdge,
                  float sInt, void* stream) {
    if (!dIn || !dOut || batch == 0 || batch > 0xFFFFFFFFull) return -8;
    if (!validShape(n, (uint32_t)batch, kExecR2C)) return -8;
    if (!pow2(n)) {   // even n, n/2 13-smooth: mixed-radix passes of n/2
        if (prepareMixed(n / 2) || prepareReal(n)) return -2;
        const auto& m = impl_->mixed[n / 2];
        if (backend::launchR2CMixed(dIn, dOut, m.plan, batch, m.tw, impl_->twReal[n], sEdge, sInt, stream)) return -5;
        return 0;
    }
    int e = 0, cta = 0;
    if (resolve(backend::kR2C, n, &e, &cta)) return -1;
    if (prepareC2C(n / 2, e) || prepareReal(n)) return -2;
    const bool weighted = !(sEdge == 1.0f && sInt == 1.0f);
    if (backend::launchR2C(dIn, dOut, n, batch, impl_->twC2C[{n / 2, e}], impl_->twReal[n], e, cta,
                           weighted, sEdge, sInt, stream))
        return -5;
    return 0;
}

int Plan::execC2R(const void* dIn, void* dOut, uint32_t n, uint64_t batch, float sEdge,
                  float sInt, float outScale, void* stream) {
    if (!dIn || !dOut || batch == 0 || batch > 0xFFFFFFFFull) return -8;
    if (!validShape(n, (uint32_t)batch, kExecC2R)) return -8;
    if (!pow2(n)) {   // even n, n/2 13-smooth: mixed-radix passes of n/2
        if (prepareMixed(n / 2) || prepareReal(n)) return -2;
        const auto& m = impl_->mixed[n / 2];
        if (backend::launchC2RMixed(dIn, dOut, m.plan, batch, m.tw, impl_->twReal[n], sEdge, sInt, outScale, stream))
            return -5;
        return 0;
    }
    int e = 0, cta = 0;
    if (resolve(backend::kC2R, n, &e, &cta)) return -1;
    if (prepareC2C(n / 2, e) || prepareReal(n)) return -2;
    if (backend::launchC2R(dIn, dOut, n, batch, impl_->twC2C[{n / 2, e}], impl_->twReal[n], e, cta,
                           sEdge, sInt, outScale, stream))
        return -5;
    return 0;
}

int Plan::execR2C2D(const void* dIn, void* dOut, uint32_t ny, uint32_t nx, uint64_t batch, float scale,
                    void* stream) {
    if (!dIn || !dOut || batch == 0 || !pow2(ny) || !backend::hasCols(ny)) return -8;
    if (batch > 0xFFFFFFFFull / ny) return -8;
    const uint32_t half = nx / 2 + 1;
    if (int r = execR2C(dIn, dOut, nx, batch * ny, 1.0f, 1.0f, stream)) return r;
    return execCols(dOut, dOut, ny, batch, half, half, false, scale, stream);
}

int Plan::execC2R2D(const void* dIn, void* dOut, uint32_t ny, uint32_t nx, uint64_t batch, float scale,
                    void* stream) {
    if (!dIn || !dOut || batch == 0 || !pow2(ny) || !backend::hasCols(ny)) return -8;
    if (batch > 0xFFFFFFFFull / ny || !validShape(nx, (uint32_t)(batch * ny), kExecC2R)) return -8;
    const uint32_t half = nx / 2 + 1;
    if (ensureBuf(&impl_->devHalf, &impl_->devHalfCap, (size_t)batch * ny * half * 8)) return -3;
    if (int r = execCols(dIn, impl_->devHalf, ny, batch, half, half, true, 1.0f, stream)) return r;
    return execC2R(impl_->devHalf, dOut, nx, batch * ny, 1.0f, 1.0f, scale, stream);
}

// Body of the synchronous host-pointer entry points: upload, enqueue, synchronise, download.
// Transfers above kPipelineBytes are cut into row chunks that flow through an upload stream, the
// context stream and a download stream, so the H2D of one chunk, the kernels of another and the
// D2H of a third overlap (two copy engines).  Chunk size trades pipeline fill against the gap
// each chunk boundary leaves on the copy engines: on B200 over PCIe 5 (99 GB/s both directions
// together) 4 MB chunks reached 81 GB/s and 16 MB chunks 92 GB/s, so a transfer is cut into
// quarters of 2..16 MB and the many-request call uses 16 MB.  enqueue() returns an exec status:
// -2 prepare and -3 alloc pass through, any other failure is a launch failure (-5).
constexpr size_t kPipelineBytes = 4u << 20, kChunkBytes = 16u << 20;
static size_t chunkBytesFor(size_t bytes) {
    return std::min<size_t>(kChunkBytes, std::max<size_t>(2u << 20, bytes / 4));
}

namespace {
// Process-wide host threads that split large copies between pageable and pinned memory (one
// thread copies about 10 GB/s; the PCIe link wants 55 GB/s per direction).
class CopyPool {
public:
    static CopyPool& get() {
        static CopyPool pool;
        return pool;
    }
    void copy(void* dst, const void* src, size_t bytes) {
        const size_t parts = std::min<size_t>(workers_.size() + 1, std::max<size_t>(1, bytes >> 20));
        if (parts <= 1) {
            std::memcpy(dst, src, bytes);
            return;
        }
        const size_t step = (bytes + parts - 1) / parts;
        std::atomic<size_t> pending{parts - 1};
        {
            std::lock_guard<std::mutex> lock(mu_);
            for (size_t p = 1; p < parts; ++p) {
                const size_t off = std::min(bytes, p * step), len = std::min(step, bytes - off);
                tasks_.push_back([=, &pending] {
                    if (len) std::memcpy(static_cast<char*>(dst) + off, static_cast<const char*>(src) + off, len);
                    if (--pending == 0) {
                        std::lock_guard<std::mutex> done(doneMu_);
                        doneCv_.notify_all();
                    }
                });
            }
        }
        cv_.notify_all();
        std::memcpy(dst, src, std::min(step, bytes));
        std::unique_lock<std::mutex> lock(doneMu_);
        doneCv_.wait(lock, [&] { return pending.load() == 0; });
    }
    ~CopyPool() {
        {
            std::lock_guard<std::mutex> lock(mu_);
            stop_ = true;
        }
        cv_.notify_all();
        for (auto& t : workers_) t.join();
    }

private:
    CopyPool() {
        const unsigned hc = std::thread::hardware_concurrency();
        const unsigned n = hc > 2 ? std::min(hc / 2, 8u) - 1 : 0;
        for (unsigned i = 0; i < n; ++i) workers_.emplace_back([this] { loop(); });
    }
    void loop() {
        for (;;) {
            std::function<void()> task;
            {
                std::unique_lock<std::mutex> lock(mu_);
                cv_.wait(lock, [&] { return stop_ || !tasks_.empty(); });
                if (stop_ && tasks_.empty()) return;
                task = std::move(tasks_.front());
                tasks_.pop_front();
            }
            task();
        }
    }
    std::vector<std::thread> workers_;
    std::deque<std::function<void()>> tasks_;
    std::mutex mu_, doneMu_;
    std::condition_variable cv_, doneCv_;
    bool stop_ = false;
};
}  // namespace

template <class Enqueue>
int Plan::roundTrip(const float* in, size_t inRowBytes, float* out, size_t outRowBytes,
                    uint32_t batch, Enqueue&& enqueue) {
    Impl* im = impl_.get();
    const size_t inBytes = inRowBytes * batch, outBytes = outRowBytes * batch;
    if (ensureBuf(&im->devIn, &im->devInCap, inBytes)) return -3;
    if (ensureBuf(&im->devOut, &im->devOutCap, outBytes)) return -3;
    bool pipelined = false;
    if (inBytes + outBytes > kPipelineBytes) {
        for (int i = 0; i < 2; ++i) {
            if (!im->aux[i] && backend::streamCreate(&im->aux[i])) im->aux[i] = nullptr;
            if (!im->ev[i] && backend::eventCreate(&im->ev[i])) im->ev[i] = nullptr;
        }
        pipelined = im->aux[0] && im->aux[1] && im->ev[0] && im->ev[1];
    }
    if (!pipelined) {   // one stream: upload, transform, download
        if (backend::copyH2D(im->devIn, in, inBytes, stream_)) return -4;
        const int lrc = enqueue(im->devIn, im->devOut, 0u, batch, stream_);
        if (lrc == -2 || lrc == -3) return lrc;
        if (lrc) return -5;
        if (backend::streamSync(stream_)) return -6;
        if (backend::copyD2H(out, im->devOut, outBytes, stream_)) return -7;
        return backend::streamSync(stream_) ? -7 : 0;
    }
    // Chunks of rows through three streams, one per stage: uploads on aux[0], transforms on the
    // context stream, downloads on aux[1], each chunk's stages ordered by two events.  Both copy
    // directions then stream back to back and overlap each other and the kernels.
    void* sIn = im->aux[0];
    void* sOut = im->aux[1];
    const size_t row = inRowBytes > outRowBytes ? inRowBytes : outRowBytes;
    const uint32_t chunk = (uint32_t)std::max<size_t>(1, chunkBytesFor(row * batch) / row);
    if (!backend::isPinnedHost(in) || !backend::isPinnedHost(out)) {
        // Pageable host buffers: the driver would stage them through its own small buffers
        // (13 GB/s here).  Instead, host threads copy each chunk into one of two pinned slots
        // while the GPU works on the previous chunk, and out of the result slot behind it.
        const size_t inChunk = (size_t)chunk * inRowBytes, outChunk = (size_t)chunk * outRowBytes;
        for (int i = 0; i < 2; ++i) {
            if (im->pinInCap < inChunk && im->pinIn[i]) {
                backend::releaseHost(im->pinIn[i]);
                im->pinIn[i] = nullptr;
            }
            if (im->pinOutCap < outChunk && im->pinOut[i]) {
                backend::releaseHost(im->pinOut[i]);
                im->pinOut[i] = nullptr;
            }
        }
        for (int i = 0; i < 2; ++i) {
            if (!im->pinIn[i] && backend::allocHost(&im->pinIn[i], std::max(inChunk, im->pinInCap))) {
                im->pinIn[i] = nullptr;
                return -3;
            }
            if (!im->pinOut[i] && backend::allocHost(&im->pinOut[i], std::max(outChunk, im->pinOutCap))) {
                im->pinOut[i] = nullptr;
                return -3;
            }
            if (!im->evStage[i] && backend::eventCreate(&im->evStage[i])) im->evStage[i] = nullptr;
            if (!im->evOut[i] && backend::eventCreate(&im->evOut[i])) im->evOut[i] = nullptr;
            if (!im->evStage[i] || !im->evOut[i]) return -3;
        }
        im->pinInCap = std::max(im->pinInCap, inChunk);
        im->pinOutCap = std::max(im->pinOutCap, outChunk);
        auto drain = [&](int code) {   // nothing may still read or fill a slot after an error
            backend::streamSync(sIn);
            backend::streamSync(stream_);
            backend::streamSync(sOut);
            return code;
        };
        CopyPool& pool = CopyPool::get();
        const uint32_t chunks = (batch + chunk - 1) / chunk;
        auto finishOut = [&](uint32_t k) -> int {
            const uint32_t r0 = k * chunk, rows = std::min(chunk, batch - r0);
            if (backend::eventSync(im->evOut[k & 1])) return -7;
            pool.copy(reinterpret_cast<char*>(out) + (size_t)r0 * outRowBytes, im->pinOut[k & 1],
                      (size_t)rows * outRowBytes);
            return 0;
        };
        for (uint32_t k = 0; k < chunks; ++k) {
            const uint32_t r0 = k * chunk, rows = std::min(chunk, batch - r0);
            const int s = (int)(k & 1);
            if (k >= 2 && backend::eventSync(im->evStage[s])) return drain(-4);   // slot s read by chunk k-2
            pool.copy(im->pinIn[s], reinterpret_cast<const char*>(in) + (size_t)r0 * inRowBytes,
                      (size_t)rows * inRowBytes);
            char* di = static_cast<char*>(im->devIn) + (size_t)r0 * inRowBytes;
            char* dout = static_cast<char*>(im->devOut) + (size_t)r0 * outRowBytes;
            if (backend::copyH2D(di, im->pinIn[s], (size_t)rows * inRowBytes, sIn)) return drain(-4);
            if (backend::eventRecord(im->evStage[s], sIn) || backend::streamWaitEvent(stream_, im->evStage[s]))
                return drain(-6);
            const int lrc = enqueue(di, dout, r0, rows, stream_);
            if (lrc == -2 || lrc == -3) return drain(lrc);
            if (lrc) return drain(-5);
            if (backend::eventRecord(im->ev[1], stream_) || backend::streamWaitEvent(sOut, im->ev[1])) return drain(-6);
            if (backend::copyD2H(im->pinOut[s], dout, (size_t)rows * outRowBytes, sOut)) return drain(-7);
            if (backend::eventRecord(im->evOut[s], sOut)) return drain(-6);
            if (k >= 1)
                if (int rc = finishOut(k - 1)) return drain(rc);
        }
        if (int rc = finishOut(chunks - 1)) return drain(rc);
        if (backend::streamSync(sIn) || backend::streamSync(stream_)) return -6;
        return backend::streamSync(sOut) ? -6 : 0;
    }
    for (uint32_t r0 = 0; r0 < batch; r0 += chunk) {
        const uint32_t rows = std::min(chunk, batch - r0);
        char* di = static_cast<char*>(im->devIn) + (size_t)r0 * inRowBytes;
        char* dout = static_cast<char*>(im->devOut) + (size_t)r0 * outRowBytes;
        if (backend::copyH2D(di, reinterpret_cast<const char*>(in) + (size_t)r0 * inRowBytes,
                             (size_t)rows * inRowBytes, sIn))
            return -4;
        if (backend::eventRecord(im->ev[0], sIn) || backend::streamWaitEvent(stream_, im->ev[0])) return -6;
        const int lrc = enqueue(di, dout, r0, rows, stream_);
        if (lrc == -2 || lrc == -3) return lrc;
        if (lrc) return -5;
        if (backend::eventRecord(im->ev[1], stream_) || backend::streamWaitEvent(sOut, im->ev[1])) return -6;
        if (backend::copyD2H(reinterpret_cast<char*>(out) + (size_t)r0 * outRowBytes, dout,
                             (size_t)rows * outRowBytes, sOut))
            return -7;
    }
    if (backend::streamSync(sIn) || backend::streamSync(stream_)) return -6;
    return backend::streamSync(sOut) ? -6 : 0;
}

int Plan::runMany(const HostRequest* reqs, size_t count) {
    if (!impl_ || !reqs || count == 0) return -8;
    constexpr size_t kAlign = 256;
    auto up = [](size_t v) { return (v + kAlign - 1) / kAlign * kAlign; };
    size_t total = 0, workElems = 0;
    for (size_t i = 0; i < count; ++i) {
        const HostRequest& r = reqs[i];
        if (!r.in || !r.out || (r.direction != -1 && r.direction != 1) || !validShape(r.n, r.batch, kExecC2C))
            return -8;
        total += up((size_t)r.n * r.batch * 8);
    }
    Impl* im = impl_.get();
    for (size_t i = 0; i < count; ++i) {   // tables, and the four-step workspace for the largest chunk
        const HostRequest& r = reqs[i];
        if (pow2(r.n) && r.n >= kMinN) {
            int e = 0, cta = 0;
            if (resolve(backend::kC2C, r.n, &e, &cta)) return -1;
            if (prepare(r.n, 1)) return -2;
            if (e == 0) {
                const size_t rows = std::min<size_t>(r.batch, std::max<size_t>(1, kChunkBytes / ((size_t)r.n * 8)));
                workElems = std::max(workElems, rows * r.n);
            }
        } else if (prepareAnyLength(r.n)) {
            return -2;
        }
    }
    if (ensureBuf(&im->devIn, &im->devInCap, total) || ensureBuf(&im->devOut, &im->devOutCap, total)) return -3;
    if (workElems && ensureBuf(&im->devWork, &im->devWorkCap, workElems * 8)) return -3;
    for (int i = 0; i < 2; ++i) {
        if (!im->aux[i] && backend::streamCreate(&im->aux[i])) im->aux[i] = nullptr;
        if (!im->ev[i] && backend::eventCreate(&im->ev[i])) im->ev[i] = nullptr;
    }
    if (!im->aux[0] || !im->aux[1] || !im->ev[0] || !im->ev[1]) return -3;
    // Row chunks of at most kChunkBytes; consecutive pieces smaller than that are grouped up to
    // kGroupBytes, each group sharing one upload event and one transform event (a group's
    // copies and kernels run as three phases, so small groups keep several in flight).
    constexpr size_t kGroupBytes = 2u << 20;
    void* sIn = im->aux[0];
    void* sOut = im->aux[1];
    struct Piece {
        const HostRequest* r;
        size_t off;   // byte offset of the piece in devIn / devOut
        uint32_t r0, rows;
    };
    std::vector<Piece> group;
    size_t groupBytes = 0;
    auto flush = [&]() -> int {
        if (group.empty()) return 0;
        for (const Piece& p : group) {
            const size_t rowBytes = (size_t)p.r->n * 8;
            if (backend::copyH2D(static_cast<char*>(im->devIn) + p.off,
                                 reinterpret_cast<const char*>(p.r->in) + (size_t)p.r0 * rowBytes,
                                 (size_t)p.rows * rowBytes, sIn))
                return -4;
        }
        if (backend::eventRecord(im->ev[0], sIn) || backend::streamWaitEvent(stream_, im->ev[0])) return -6;
        for (const Piece& p : group) {
            const int lrc = execC2CWith(static_cast<char*>(im->devIn) + p.off, static_cast<char*>(im->devOut) + p.off,
                                        p.r->n, p.rows, p.r->direction, p.r->scale, stream_, im->devWork);
            if (lrc == -2 || lrc == -3) return lrc;
            if (lrc) return -5;
        }
        if (backend::eventRecord(im->ev[1], stream_) || backend::streamWaitEvent(sOut, im->ev[1])) return -6;
        for (const Piece& p : group) {
            const size_t rowBytes = (size_t)p.r->n * 8;
            if (backend::copyD2H(reinterpret_cast<char*>(p.r->out) + (size_t)p.r0 * rowBytes,
                                 static_cast<char*>(im->devOut) + p.off, (size_t)p.rows * rowBytes, sOut))
                return -7;
        }
        group.clear();
        groupBytes = 0;
        return 0;
    };
    // Issue order: requests under 1 MB first, then every other remaining request by size
    // (smallest first), the rest last (largest first), so the largest requests stream in the
    // middle and both ends of the
    // pipeline are short; near the end pieces shrink to half of what is left (at least
    // 512 KB), so the final download trailing the last upload is short.  Measured over the
    // 49-point grid with pinned buffers: +2 % against request order and fixed 16 MB pieces;
    // smaller fixed pieces lose (each copy costs microseconds of its own).
    std::vector<size_t> offs(count), bySize(count), order;
    size_t remaining = 0;
    for (size_t i = 0, off = 0; i < count; ++i) {
        offs[i] = off;
        off += up((size_t)reqs[i].n * reqs[i].batch * 8);
        remaining += (size_t)reqs[i].n * reqs[i].batch * 8;
        bySize[i] = i;
    }
    auto bytesOf = [&](size_t i) { return (size_t)reqs[i].n * reqs[i].batch * 8; };
    std::stable_sort(bySize.begin(), bySize.end(), [&](size_t a, size_t b) { return bytesOf(a) < bytesOf(b); });
    // Requests below kSmallBytes all go first: their copies cost about their latency (~10 us
    // each), which the first large uploads hide, whereas at the end of the pipeline they would
    // run one after another behind the last upload.
    constexpr size_t kSmallBytes = 1u << 20;
    size_t small = 0;
    while (small < count && bytesOf(bySize[small]) < kSmallBytes) order.push_back(bySize[small++]);
    const size_t large = count - small;
    for (size_t k = 0; k < large; k += 2) order.push_back(bySize[small + k]);
    for (size_t k = large - 1 - (large % 2 == 0 ? 0 : 1); k < large; k -= 2) order.push_back(bySize[small + k]);
    for (const size_t i : order) {
        const HostRequest& r = reqs[i];
        const size_t rowBytes = (size_t)r.n * 8;
        for (uint32_t r0 = 0; r0 < r.batch;) {
            const size_t want = std::min<size_t>(kChunkBytes, std::max<size_t>(512u << 10, remaining / 2));
            const uint32_t rows = (uint32_t)std::min<size_t>(r.batch - r0, std::max<size_t>(1, want / rowBytes));
            group.push_back({&r, offs[i] + (size_t)r0 * rowBytes, r0, rows});
            groupBytes += (size_t)rows * rowBytes;
            remaining -= (size_t)rows * rowBytes;
            r0 += rows;
            if (groupBytes >= kGroupBytes)
                if (int rc = flush()) return rc;
        }
    }
    if (int rc = flush()) return rc;
    if (backend::streamSync(sIn) || backend::streamSync(stream_)) return -6;
    return backend::streamSync(sOut) ? -6 : 0;
}

int Plan::run(const float* in, float* out, uint32_t n, uint32_t batch) {
    if (!in || !out || !validShape(n, batch, kRunC2C)) return -8;
    if (prepare(n, batch)) return -2;
    return roundTrip(in, (size_t)n * 8, out, (size_t)n * 8, batch,
                     [&](void* di, void* dout, uint32_t, uint32_t rows, void* st) {
                         return execC2C(di, dout, n, rows, -1, 1.0f, st);
                     });
}

int Plan::runInverse(const float* in, float* out, uint32_t n, uint32_t batch, float scale) {
    if (!in || !out || !validShape(n, batch, kRunC2C)) return -8;
    if (prepare(n, batch)) return -2;
    return roundTrip(in, (size_t)n * 8, out, (size_t)n * 8, batch,
                     [&](void* di, void* dout, uint32_t, uint32_t rows, void* st) {
                         return execC2C(di, dout, n, rows, 1, scale, st);
                     });
}

int Plan::runLong(const float* in, float* out, uint32_t n, uint32_t batch, int direction) {
    if (!in || !out || (direction != -1 && direction != 1) || !validShape(n, batch, kRunLong)) return -8;
    if (prepare(n, batch)) return -2;
    int e = 0, cta = 0;
    if (resolve(backend::kC2C, n, &e, &cta)) return -1;
    if (e == 0 && ensureBuf(&impl_->devWork, &impl_->devWorkCap, (size_t)n * batch * 8)) return -3;
    // chunks on different streams use disjoint slices of the four-step workspace
    return roundTrip(in, (size_t)n * 8, out, (size_t)n * 8, batch,
                     [&](void* di, void* dout, uint32_t r0, uint32_t rows, void* st) {
                         void* work = e != 0 ? nullptr : static_cast<char*>(impl_->devWork) + (size_t)r0 * n * 8;
                         return execC2CWith(di, dout, n, rows, direction, 1.0f, st, work);
                     });
}

int Plan::runR2C(const float* in, float* out, uint32_t n, uint32_t batch) {
    if (!in || !out || !validShape(n, batch, kRunR2C)) return -8;
    int e = 0, cta = 0;
    if (resolve(backend::kR2C, n, &e, &cta)) return -1;
    if (prepareC2C(n / 2, e) || prepareReal(n)) return -2;
    return roundTrip(in, (size_t)n * 4, out, (size_t)(n + 2) * 4, batch,
                     [&](void* di, void* dout, uint32_t, uint32_t rows, void* st) {
                         return execR2C(di, dout, n, rows, 1.0f, 1.0f, st);
                     });
}

int Plan::runC2R(const float* in, float* out, uint32_t n, uint32_t batch) {
    if (!in || !out || !validShape(n, batch, kRunC2R)) return -8;
    int e = 0, cta = 0;
    if (resolve(backend::kC2R, n, &e, &cta)) return -1;
    if (prepareC2C(n / 2, e) || prepareReal(n)) return -2;
    return roundTrip(in, (size_t)(n + 2) * 4, out, (size_t)n * 4, batch,
                     [&](void* di, void* dout, uint32_t, uint32_t rows, void* st) {
                         return execC2R(di, dout, n, rows, 1.0f, 1.0f, 1.0f / (float)n, st);
                     });
}

int Plan::measure(uint32_t n, uint32_t batch, Metric* m) {
    if (!m) return -1;
    if (!validShape(n, batch, kMeasure)) return -8;
    const size_t nf = (size_t)n * 2 * batch;
    std::vector<float> in(nf), out(nf);
    for (size_t i = 0; i < nf; ++i) in[i] = patternAt(i);
    if (prepare(n, batch)) return -2;
    const int first = roundTrip(in.data(), (size_t)n * 8, out.data(), (size_t)n * 8, batch,
                                [&](void* di, void* dout, uint32_t, uint32_t rows, void* st) {
                                    return execC2C(di, dout, n, rows, -1, 1.0f, st);
                                });
    if (first) return -2;
    if (!impl_->timer && backend::timerCreate(&impl_->timer)) return -3;
    // Device time per launch (CUDA events on the plan stream): a chain of back-to-back launches
    // lasting ~50 us -- the steady state of repeated calls, and well above the events'
    // resolution for microsecond kernels, whose single launches rank by launch jitter --
    // best of 5 chains.
    auto chain = [&](int reps, float* ms) -> int {
        if (backend::timerStart(impl_->timer, stream_)) return -3;
        for (int i = 0; i < reps; ++i)
            if (execC2C(impl_->devIn, impl_->devOut, n, batch, -1, 1.0f, stream_)) return -4;
        if (backend::timerStop(impl_->timer, stream_, ms)) return -3;
        return 0;
    };
    float ms = 0.f;
    if (int r = chain(1, &ms)) return r;   // warm-up
    if (int r = chain(1, &ms)) return r;
    const int reps = std::max(1, std::min(64, (int)(0.05 / std::max(ms, 1e-4f))));
    double best = 0.0;
    for (int r = 0; r < 5; ++r) {
        if (int e = chain(reps, &ms)) return e == -4 ? -5 : e;
        const double us = ms * 1000.0 / reps;
        if (r == 0 || us < best) best = us;
    }
    m->measuredUs = best;
    if (backend::copyD2H(out.data(), impl_->devOut, nf * 4, stream_) || backend::streamSync(stream_)) return -6;
    m->etaUs = cand_.q.etaUs;
    uint32_t idx[8];
    const uint32_t cnt = sampleBatches(batch, 8, idx, 8);
    std::vector<float> ref(2 * (size_t)n);
    double maxRel = 0.0;
    for (uint32_t i = 0; i < cnt; ++i) {
        const size_t off = (size_t)idx[i] * 2 * n;
        refFftF32(in.data() + off, ref.data(), n);
        maxRel = std::max(maxRel, maxRelScaled(out.data() + off, ref.data(), 2 * (size_t)n));
    }
    m->maxRelErr = maxRel;
    if (!std::isfinite(maxRel) || maxRel > 1e-4) {
        m->measuredOk = false;
        cand_.q = *m;
        cand_.state = State::Unverified;
        cand_.reason = "correctness check failed (maxRel > 1e-4)";
        return -7;
    }
    m->measuredOk = true;
    cand_.q = *m;
    cand_.reason.clear();
    cand_.state = State::Measured;
    return 0;
}

// ================================================================== ragged
Ragged::~Ragged() {
    if (entries_) backend::release(entries_);
    if (tileMap_) backend::release(tileMap_);
}

int Ragged::exec(void* stream) const {
    const int r = stages_ < 0   ? backend::launchRaggedFlat(entries_, (int)count_, tileMap_, total_, stream)
                  : stages_ > 0 ? backend::launchRaggedStaged(entries_, (int)count_, total_, grid_, stages_, stream)
                                : backend::launchRagged(entries_, (int)count_, total_, grid_, stream);
    return r ? -5 : 0;
}

int Ragged::deviceStatus(unsigned* status) {
    if (!status) return -10;
    return backend::raggedStatus(status, true) ? -6 : 0;
}

static_assert(RaggedConfig{}.radix8 == kRaggedDefaultRadix8, "default ragged radices differ");

std::unique_ptr<Ragged> Plan::makeRagged(const RaggedRequest* reqs, size_t count, int* status,
                                         const RaggedConfig* config) {
    int dummy = 0;
    int& st = status ? *status : dummy;
    st = -8;
    if (!impl_ || !reqs || count == 0 || count > (1u << 24)) return nullptr;
    for (size_t i = 0; i < count; ++i) {
        const RaggedRequest& r = reqs[i];
        if (!r.in || !r.out || !pow2(r.n) || r.n < kRaggedMinN || r.n > kRaggedMaxN || r.batch == 0 ||
            (r.direction != -1 && r.direction != 1))
            return nullptr;
    }
    bool aligned = true;
    for (size_t i = 0; i < count; ++i) aligned = aligned && ((uintptr_t)reqs[i].in % 16u) == 0;
    RaggedConfig cfg;
    if (config) {
        cfg = *config;
        if (cfg.mode < -1 || cfg.mode > 2 || (cfg.mode > 0 && !aligned) ||
            (cfg.radix8 >> (kRaggedMaxLog - kRaggedMinLog)) != 0)
            return nullptr;
    } else {
        cfg.mode = -1;   // one tile per CTA: measured fastest on B200 (hardware CTA scheduling)
        if (const char* env = std::getenv("BFLY_RAGGED_STAGES")) {
            const int want = std::atoi(env);
            if (want >= -1 && want <= 2) cfg.mode = (aligned || want < 0) ? want : 0;
        }
    }
    std::vector<RaggedEntry> es(count);
    uint64_t tile = 0;
    for (size_t i = 0; i < count; ++i) {
        const RaggedRequest& r = reqs[i];
        int logn = 0;
        while ((1u << logn) < r.n) ++logn;
        const int e = (cfg.radix8 >> (logn - kRaggedMinLog)) & 1u ? 8 : 16;
        if (!raggedVariant(logn, e)) return nullptr;
        if (prepareC2C(r.n, e)) {
            st = -2;
            return nullptr;
        }
        const uint32_t rows = raggedRows(logn, e);
        es[i] = RaggedEntry{r.in, r.out, impl_->twC2C[{r.n, e}], r.batch, tile, (uint32_t)logn,
                            r.direction, r.scale, rows, (uint32_t)e, 0};
        tile += (r.batch + rows - 1) / rows;
    }
    std::unique_ptr<Ragged> rg(new Ragged());
    rg->count_ = count;
    rg->total_ = tile;
    rg->stages_ = cfg.mode;
    rg->radix8_ = cfg.radix8;
    rg->aligned_ = aligned;
    const int grc = rg->stages_ > 0 ? backend::raggedStagedGrid(impl_->device, rg->stages_, &rg->grid_)
                                    : backend::raggedGrid(impl_->device, &rg->grid_);
    if (grc) {
        st = -1;
        return nullptr;
    }
    if (backend::alloc(&rg->entries_, count * sizeof(RaggedEntry))) {
        rg->entries_ = nullptr;
        st = -3;
        return nullptr;
    }
    if (backend::copyH2D(rg->entries_, es.data(), count * sizeof(RaggedEntry), stream_)) {
        st = -4;
        return nullptr;
    }
    // request index of every tile for the one-tile-per-CTA mode (up to 4 Mi tiles = 16 MiB;
    // larger work lists fall back to a binary search per CTA)
    std::vector<uint32_t> map;
    if (rg->stages_ < 0 && tile <= (4ull << 20)) {
        map.resize(tile);
        for (size_t i = 0; i < count; ++i) {
            const uint64_t end = i + 1 < count ? es[i + 1].tile0 : tile;
            for (uint64_t t = es[i].tile0; t < end; ++t) map[t] = (uint32_t)i;
        }
        if (backend::alloc(&rg->tileMap_, map.size() * sizeof(uint32_t))) {
            rg->tileMap_ = nullptr;
            st = -3;
            return nullptr;
        }
        if (backend::copyH2D(rg->tileMap_, map.data(), map.size() * sizeof(uint32_t), stream_)) {
            st = -4;
            return nullptr;
        }
    }
    if (backend::streamSync(stream_)) {
        st = -4;
        return nullptr;
    }
    st = 0;
    return rg;
}

double Plan::timeRagged(const Ragged& rg) {
    if (!impl_) return -1.0;
    if (!impl_->timer && backend::timerCreate(&impl_->timer)) return -3.0;
    auto chain = [&](int reps, float* ms) -> int {
        if (backend::timerStart(impl_->timer, stream_)) return -3;
        for (int i = 0; i < reps; ++i)
            if (rg.exec(stream_)) return -5;
        if (backend::timerStop(impl_->timer, stream_, ms)) return -3;
        return 0;
    };
    float ms = 0.f;
    if (int r = chain(1, &ms)) return r;
    if (int r = chain(1, &ms)) return r;
    const int reps = std::max(1, std::min(64, (int)(1.0 / std::max(ms, 1e-4f))));
    // ~3 ms of back-to-back launches first: after the host-side gaps of the caller (work list
    // builds, synchronisations) the device runs this kernel a few percent slower for the
    // first milliseconds
    if (int r = chain(std::min(256, 3 * reps), &ms)) return r;
    double best = 0.0;
    for (int r = 0; r < 3; ++r) {
        if (int e = chain(reps, &ms)) return e;
        const double us = ms * 1000.0 / reps;
        if (r == 0 || us < best) best = us;
    }
    return best;
}

// ================================================================== Context
struct Context::Impl {
    void* stream = nullptr;
    bool initialized = false;
};

Context::Context() : impl_(new Impl) {}

Context::~Context() {
    if (impl_->stream) backend::streamDestroy(impl_->stream);
}

void* Context::stream() const { return impl_->stream; }

int Context::init(const std::string& profilePath, const std::string& spacePath,
                  const std::string& kernelPath) {
    return init(profilePath, spacePath, kernelPath, -1);
}

int Context::init(const std::string& profilePath, const std::string& spacePath,
                  const std::string& kernelPath, int device) {
    if (impl_->initialized) return -9;
    Hardware hardware;
    DesignSpace space;
    try {
        hardware = Hardware::load(profilePath);
        space = DesignSpace::load(spacePath);
    } catch (const std::exception& e) {
        std::fprintf(stderr, "Context::init configuration error: %s\n", e.what());
        return -4;
    }
    hw_ = std::move(hardware);
    sp_ = std::move(space);
    kernelPath_ = kernelPath;
    if (device >= 0) hw_.deviceIndex = device;
    int count = 0;
    if (backend::deviceCount(&count) || count <= 0) return -1;
    if (hw_.deviceIndex >= count || backend::setDevice(hw_.deviceIndex)) return -2;
    if (backend::streamCreate(&impl_->stream)) return -3;
    impl_->initialized = true;
    return 0;
}

std::vector<Candidate> Context::enumerate(uint32_t n, uint32_t batch) const {
    return bfly::enumerate(sp_, hw_, n, batch);
}

std::unique_ptr<Plan> Context::makePlan(const Candidate& c) {
    if (!impl_->initialized || c.state == State::Infeasible || !lowerable(c, hw_)) return nullptr;
    if (!kernelPath_.empty() && kernelPath_ != "builtin") {
        std::ifstream f(kernelPath_, std::ios::binary);
        if (!f) return nullptr;   // the named kernel library does not exist
    }
    auto p = std::unique_ptr<Plan>(new Plan(c));
    p->impl_.reset(new Plan::Impl());
    p->impl_->hw = hw_;
    p->impl_->device = hw_.deviceIndex;
    p->stream_ = impl_->stream;
    p->tf_.push_back({Transform::GenTwiddles, "FP64 twiddle tables built on the device, rounded to fp32"});
    p->tf_.push_back({Transform::LaunchKernel, "hand-written sm_100a kernels on the context stream"});
    return p;
}

// ------------------------------------------------------------------ tuning cache
namespace {
struct CacheEntry {
    std::string gpu, kind, id;
    long long n = 0, batch = 0;
    double us = 0.0;
};

std::vector<CacheEntry> readCache(const std::string& path) {
    std::vector<CacheEntry> out;
    std::ifstream f(path, std::ios::binary);
    if (!f) return out;
    try {
        const std::string text((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
        const json::Node root = json::parse(text);
        if (root.get("schema_version").asInt() != 1) return out;
        for (const auto& e : root.get("entries").items) {
            CacheEntry c;
            c.gpu = e.get("gpu").asString();
            c.kind = e.get("kind").asString();
            c.id = e.get("id").asString();
            c.n = e.get("n").asInt();
            c.batch = e.get("batch").asInt();
            c.us = e.get("us").asDouble();
            out.push_back(c);
        }
    } catch (const std::exception&) {
        out.clear();   // an unreadable cache is ignored and rewritten
    }
    return out;
}

std::string escapeJson(const std::string& s) {
    std::string o;
    for (char ch : s) {
        if (ch == '"' || ch == '\\') o += '\\';
        if ((unsigned char)ch >= 0x20) o += ch;
    }
    return o;
}

void writeCache(const std::string& path, const std::vector<CacheEntry>& es) {
    std::ostringstream os;
    os << "{\n  \"schema_version\": 1,\n  \"entries\": [";
    for (size_t i = 0; i < es.size(); ++i) {
        const auto& e = es[i];
        char us[64];
        std::snprintf(us, sizeof(us), "%.3f", e.us);
        os << (i ? ",\n" : "\n") << "    {\"gpu\": \"" << escapeJson(e.gpu) << "\", \"kind\": \""
           << escapeJson(e.kind) << "\", \"n\": " << e.n << ", \"batch\": " << e.batch
           << ", \"id\": \"" << escapeJson(e.id) << "\", \"us\": " << us << "}";
    }
    os << "\n  ]\n}\n";
    const std::string tmp = path + ".tmp";
    {
        std::ofstream f(tmp, std::ios::binary | std::ios::trunc);
        if (!f) return;
        f << os.str();
        if (!f) return;
    }
    std::rename(tmp.c_str(), path.c_str());
}
}  // namespace

std::unique_ptr<Plan> Context::select(uint32_t n, uint32_t batch, int topK, std::string* log) {
    auto all = enumerate(n, batch);
    auto order = rank(all);
    const int k = std::max(1, topK);
    char line[512];
    if (log) {
        log->clear();
        int infeasible = 0;
        for (const auto& c : all) infeasible += c.state == State::Infeasible;
        std::snprintf(line, sizeof(line), "enumerated=%zu infeasible=%d feasible=%zu (n=%u batch=%u)\n",
                      all.size(), infeasible, order.size(), n, batch);
        *log += line;
        std::vector<std::pair<int, std::string>> reasons;
        for (const auto& c : all) {
            if (c.state != State::Infeasible) continue;
            bool hit = false;
            for (auto& r : reasons)
                if (r.second == c.reason) { ++r.first; hit = true; break; }
            if (!hit) reasons.push_back({1, c.reason});
        }
        std::stable_sort(reasons.begin(), reasons.end(), [](auto& x, auto& y) { return x.first > y.first; });
        for (size_t i = 0; i < reasons.size() && i < 5; ++i) {
            std::snprintf(line, sizeof(line), "  infeasible x%-4d %s\n", reasons[i].first, reasons[i].second.c_str());
            *log += line;
        }
        std::snprintf(line, sizeof(line), "  eta rank (top %d):\n", k);
        *log += line;
        for (size_t i = 0; i < order.size() && i < (size_t)k; ++i) {
            std::snprintf(line, sizeof(line), "    %2zu. %-44s eta=%8.1f us  [%s]\n", i + 1,
                          order[i]->id.c_str(), order[i]->q.etaUs, toString(order[i]->state));
            *log += line;
        }
    }
    if (order.empty()) return nullptr;

    // Persisted choice for this (gpu, n, batch)?
    std::vector<CacheEntry> cache;
    if (!tuningCache_.empty()) {
        cache = readCache(tuningCache_);
        for (const auto& e : cache) {
            if (e.gpu != hw_.gpu || e.kind != "c2c" || e.n != n || e.batch != batch) continue;
            for (const Candidate* c : order) {
                if (c->id != e.id) continue;
                auto p = makePlan(*c);
                if (p) {
                    if (log) {
                        std::snprintf(line, sizeof(line), "  selected: %s  (tuning cache, %.1f us)\n", c->id.c_str(), e.us);
                        *log += line;
                    }
                    return p;
                }
            }
        }
    }

    if (log) *log += "  measured selection:\n";
    std::unique_ptr<Plan> best;
    double bestUs = 0.0;
    int measured = 0;
    size_t examined = 0;
    for (size_t i = 0; i < order.size() && measured < k; ++i) {
        ++examined;
        const Candidate& c = *order[i];
        auto p = makePlan(c);
        if (!p) {
            if (log) {
                std::snprintf(line, sizeof(line), "    fail   %-44s eta=%8.1f us  makePlan failed\n", c.id.c_str(), c.q.etaUs);
                *log += line;
            }
            continue;
        }
        Metric m;
        const int rc = p->measure(n, batch, &m);
        if (rc) {
            if (log) {
                std::snprintf(line, sizeof(line), "    reject %-44s eta=%8.1f us  rc=%d maxRel=%.2e  [%s]\n",
                              c.id.c_str(), c.q.etaUs, rc, m.maxRelErr, toString(p->candidate().state));
                *log += line;
            }
            continue;
        }
        ++measured;
        if (log) {
            std::snprintf(line, sizeof(line), "    accept %-44s eta=%8.1f us  measured=%8.1f us  maxRel=%.1e  [%s]\n",
                          p->candidate().id.c_str(), m.etaUs, m.measuredUs, m.maxRelErr,
                          toString(p->candidate().state));
            *log += line;
        }
        if (!best || m.measuredUs < bestUs) {
            bestUs = m.measuredUs;
            best = std::move(p);
        }
    }
    if (log) {
        if (best)
            std::snprintf(line, sizeof(line), "  selected: %s  (%.1f us, %d accepted after %zu examined, quota %d)\n",
                          best->candidate().id.c_str(), bestUs, measured, examined, k);
        else
            std::snprintf(line, sizeof(line), "  selected: none (%d accepted after %zu examined, quota %d)\n",
                          measured, examined, k);
        *log += line;
    }
    if (best && !tuningCache_.empty()) {
        cache.erase(std::remove_if(cache.begin(), cache.end(), [&](const CacheEntry& e) {
                        return e.gpu == hw_.gpu && e.kind == "c2c" && e.n == n && e.batch == batch;
                    }), cache.end());
        cache.push_back({hw_.gpu, "c2c", best->candidate().id, (long long)n, (long long)batch, bestUs});
        writeCache(tuningCache_, cache);
    }
    return best;
}

namespace {
// Key of a ragged work list's shape: lengths and batch counts in order, and whether every input
// is 16-byte aligned (the staged modes need it).  Pointers, directions and scales do not change
// the launch cost and are left out.  FNV-1a, 64 bits.
uint64_t raggedShapeHash(const RaggedRequest* reqs, size_t count, bool aligned) {
    uint64_t h = 1469598103934665603ull;
    auto mix = [&](uint64_t v) {
        for (int i = 0; i < 8; ++i) {
            h ^= (v >> (8 * i)) & 0xFFu;
            h *= 1099511628211ull;
        }
    };
    mix(count);
    mix(aligned ? 1 : 0);
    for (size_t i = 0; i < count; ++i) {
        mix(reqs[i].n);
        mix(reqs[i].batch);
    }
    return h;
}

std::string raggedCacheId(uint64_t hash, const RaggedConfig& c) {
    char buf[96];
    std::snprintf(buf, sizeof(buf), "h%016llx mode %d radix8 0x%02x", (unsigned long long)hash, c.mode,
                  (unsigned)c.radix8);
    return buf;
}

bool parseRaggedCacheId(const std::string& id, uint64_t* hash, RaggedConfig* c) {
    unsigned long long h = 0;
    int mode = 0;
    unsigned mask = 0;
    if (std::sscanf(id.c_str(), "h%16llx mode %d radix8 0x%x", &h, &mode, &mask) != 3) return false;
    *hash = h;
    c->mode = mode;
    c->radix8 = mask;
    return true;
}
}  // namespace

std::unique_ptr<Ragged> Context::tuneRagged(Plan& plan, const RaggedRequest* reqs, size_t count, int* status,
                                            std::string* log) {
    int dummy = 0;
    int& st = status ? *status : dummy;
    char line[256];
    if (log) log->clear();
    // the default build validates the requests and tells the alignment
    std::unique_ptr<Ragged> best = plan.makeRagged(reqs, count, &st, nullptr);
    if (!best) return nullptr;
    if (best->stages() != -1) {   // an environment override of the mode: start from the default
        RaggedConfig def;
        best = plan.makeRagged(reqs, count, &st, &def);
        if (!best) return nullptr;
    }
    const bool aligned = best->aligned();
    const uint64_t hash = raggedShapeHash(reqs, count, aligned);
    uint64_t rows = 0;
    for (size_t i = 0; i < count; ++i) rows += reqs[i].batch;

    std::vector<CacheEntry> cache;
    if (!tuningCache_.empty()) {
        cache = readCache(tuningCache_);
        for (const auto& e : cache) {
            uint64_t h = 0;
            RaggedConfig c;
            if (e.gpu != hw_.gpu || e.kind != "ragged" || e.n != (long long)count || e.batch != (long long)rows ||
                !parseRaggedCacheId(e.id, &h, &c) || h != hash)
                continue;
            int cst = 0;
            auto rg = plan.makeRagged(reqs, count, &cst, &c);
            if (rg) {
                if (log) {
                    std::snprintf(line, sizeof(line), "selected: mode %d radix8 0x%02x (tuning cache, %.1f us)\n",
                                  c.mode, (unsigned)c.radix8, e.us);
                    *log += line;
                }
                st = 0;
                return rg;
            }
        }
    }

    double bestUs = plan.timeRagged(*best);
    if (bestUs < 0) {
        st = -5;
        return nullptr;
    }
    if (log) {
        std::snprintf(line, sizeof(line), "requests=%zu rows=%llu tiles=%llu aligned=%d\n", count,
                      (unsigned long long)rows, (unsigned long long)best->tiles(), aligned ? 1 : 0);
        *log += line;
        std::snprintf(line, sizeof(line), "  mode %2d radix8 0x%02x  %9.2f us  (default)\n", best->stages(),
                      (unsigned)best->config().radix8, bestUs);
        *log += line;
    }
    // A candidate is timed next to the incumbent in the order candidate, incumbent, incumbent,
    // candidate and each is the mean of its two timings: the device's speed drifts by a few
    // percent over seconds of intermittent load, and this order cancels a drift that is linear
    // over the four.  A step in that speed can still favour one side of a comparison, so a
    // candidate that wins by >= 1% is compared once more and replaces the incumbent only if it
    // wins again.
    auto compare = [&](const Ragged& cand, double* us, double* inc) -> int {
        const double a0 = plan.timeRagged(cand);
        const double b0 = plan.timeRagged(*best);
        const double b1 = plan.timeRagged(*best);
        const double a1 = plan.timeRagged(cand);
        if (a0 < 0 || a1 < 0 || b0 < 0 || b1 < 0) return -5;
        *us = 0.5 * (a0 + a1);
        *inc = 0.5 * (b0 + b1);
        return 0;
    };
    auto tryConfig = [&](const RaggedConfig& c) -> int {
        int cst = 0;
        auto rg = plan.makeRagged(reqs, count, &cst, &c);
        if (!rg) return cst ? cst : -1;
        double us = 0.0;
        if (compare(*rg, &us, &bestUs)) return -5;
        bool better = us < bestUs * 0.99;
        double us2 = 0.0, inc2 = 0.0;
        if (better) {
            if (compare(*rg, &us2, &inc2)) return -5;
            better = us2 < inc2 * 0.99;
        }
        unsigned dstat = 0;
        if (c.mode > 0 && (Ragged::deviceStatus(&dstat) || dstat)) {   // a bounded wait gave up
            if (log) {
                std::snprintf(line, sizeof(line), "  mode %2d radix8 0x%02x  rejected (device status %u)\n",
                              c.mode, (unsigned)c.radix8, dstat);
                *log += line;
            }
            return 0;
        }
        if (log) {
            if (us2 > 0.0)
                std::snprintf(line, sizeof(line),
                              "  mode %2d radix8 0x%02x  %9.2f us  (incumbent %.2f us; again %.2f vs %.2f)%s\n",
                              c.mode, (unsigned)c.radix8, us, bestUs, us2, inc2, better ? "  <- best" : "");
            else
                std::snprintf(line, sizeof(line), "  mode %2d radix8 0x%02x  %9.2f us  (incumbent %.2f us)\n",
                              c.mode, (unsigned)c.radix8, us, bestUs);
            *log += line;
        }
        if (better) {
            best = std::move(rg);
            bestUs = us2;
        }
        return 0;
    };
    // lengths present, largest share of points first
    uint64_t points[kRaggedMaxLog + 1] = {};
    for (size_t i = 0; i < count; ++i) {
        int logn = 0;
        while ((1u << logn) < reqs[i].n) ++logn;
        points[logn] += reqs[i].batch * reqs[i].n;
    }
    std::vector<int> lengths;
    for (int l = kRaggedMinLog; l <= kRaggedMaxLog; ++l)
        if (points[l] && raggedVariant(l, 8)) lengths.push_back(l);
    std::stable_sort(lengths.begin(), lengths.end(), [&](int a, int b) { return points[a] > points[b]; });
    for (int l : lengths) {
        RaggedConfig c = best->config();
        c.radix8 ^= 1u << (l - kRaggedMinLog);
        if (int r = tryConfig(c)) {
            st = r;
            return nullptr;
        }
    }
    for (int mode : {0, 1, 2}) {
        if (mode > 0 && !aligned) continue;
        RaggedConfig c = best->config();
        if (c.mode == mode) continue;
        c.mode = mode;
        if (int r = tryConfig(c)) {
            st = r;
            return nullptr;
        }
    }
    if (log) {
        std::snprintf(line, sizeof(line), "selected: mode %d radix8 0x%02x  %.2f us\n", best->stages(),
                      (unsigned)best->config().radix8, bestUs);
        *log += line;
    }
    if (!tuningCache_.empty()) {
        cache.erase(std::remove_if(cache.begin(), cache.end(), [&](const CacheEntry& e) {
                        uint64_t h = 0;
                        RaggedConfig c;
                        return e.gpu == hw_.gpu && e.kind == "ragged" && e.n == (long long)count &&
                               e.batch == (long long)rows && parseRaggedCacheId(e.id, &h, &c) && h == hash;
                    }), cache.end());
        cache.push_back({hw_.gpu, "ragged", raggedCacheId(hash, best->config()), (long long)count, (long long)rows,
                         bestUs});
        writeCache(tuningCache_, cache);
    }
    st = 0;
    return best;
}

}  // namespace bfly
