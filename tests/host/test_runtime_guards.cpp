// CPU host-runtime tests against the fake device seam (fake_backend.cpp).  Ports the intent of
// the reference's tests/test_runtime_guards.cpp: strict configuration loading, -9 re-init,
// candidate mutations that have no lowering, guards that reject every illegal shape with zero
// allocations / copies / launches, and failure injection proving a failed prepare never leaves
// a stale key.  Adds the B200 runtime's own contracts: host round-trip error codes, measure and
// select acceptance, and the persisted tuning cache.
#include "backend.h"
#include "bfly/plan.hpp"

#include <algorithm>
#include <cassert>
#include <cmath>
#include <cstdio>
#include <initializer_list>
#include <cstring>
#include <fstream>
#include <functional>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

namespace fake {
extern int allocations, releases, copies, launches, syncs;
extern int failAllocation, failCopy, failLaunch, failSync;
extern int streamsCreated, streamsDestroyed, deviceCountValue;
extern float timerMs;
extern int timedExtra, raggedCost16;
extern bool pageableHost;
extern std::vector<const void*> h2dSources;
}  // namespace fake

#define CHECK(cond)                                                                    \
    do {                                                                               \
        if (!(cond)) {                                                                 \
            std::fprintf(stderr, "CHECK failed at %s:%d: %s\n", __FILE__, __LINE__, #cond); \
            std::exit(1);                                                              \
        }                                                                              \
    } while (0)

static std::string read(const std::string& path) {
    std::ifstream f(path);
    return {std::istreambuf_iterator<char>(f), std::istreambuf_iterator<char>()};
}
static std::string replaced(std::string text, const std::string& from, const std::string& to) {
    const size_t at = text.find(from);
    CHECK(at != std::string::npos);
    text.replace(at, from.size(), to);
    return text;
}
static void write(const std::string& path, const std::string& text) {
    std::ofstream f(path);
    f << text;
    CHECK(f.good());
}
static bool throws(const std::function<void()>& fn) {
    try {
        fn();
    } catch (const std::exception&) {
        return true;
    }
    return false;
}

int main(int argc, char** argv) {
    CHECK(argc == 3);
    const std::string cfg = argv[1], tmp = argv[2];
    const std::string profile = cfg + "/b200_profile.json", space = cfg + "/b200_space.json";
    const std::string hwText = read(profile), spText = read(space);
    const std::string badHw = tmp + "/hw.json", badSp = tmp + "/space.json";

    // ---- strict configuration (-4), no runtime touched
    CHECK(throws([] { bfly::Hardware::load("/nonexistent-hardware-config"); }));
    CHECK(throws([] { bfly::DesignSpace::load("/nonexistent-space-config"); }));
    for (const auto& bad : {std::string("{}"), hwText + " trailing",
                            replaced(hwText, "\"sm_count\": 148", "\"sm_count\": 0"),
                            replaced(hwText, "\"sm_count\": 148", "\"sm_count\": \"148\""),
                            replaced(hwText, "\"sm_count\": 148", "\"sm_count\": 148.5"),
                            replaced(hwText, "\"hbm_gbs\": 6446.0", "\"hbm_gbs\": -1"),
                            replaced(hwText, "\"schema_version\": 1", "\"schema_version\": 2"),
                            replaced(hwText, "\"sm_count\": 148,", "\"sm_count\": 148, \"sm_count\": 1,")}) {
        write(badHw, bad);
        CHECK(throws([&] { bfly::Hardware::load(badHw); }));
        bfly::Context invalid;
        CHECK(invalid.init(badHw, space, "builtin") == -4);
    }
    for (const auto& bad : {std::string("{"), std::string("{}"), spText + " trailing",
                            replaced(spText, "\"cta_threads\": [128, 256, 512, 1024]", "\"cta_threads\": []"),
                            replaced(spText, "\"cta_threads\": [128, 256, 512, 1024]", "\"cta_threads\": [100]"),
                            replaced(spText, "\"radix\": [8, 16]", "\"radix\": [\"8\"]"),
                            replaced(spText, "\"radix\": [8, 16]", "\"radix\": [3]"),
                            replaced(spText, "\"out\": [\"interleaved\", \"planar\"]", "\"out\": [\"bogus\"]"),
                            replaced(spText, "\"schedule\": [\"stockham\", \"cluster\", \"four_step\", \"ring\"]", "\"schedule\": [\"fast\"]")}) {
        write(badSp, bad);
        CHECK(throws([&] { bfly::DesignSpace::load(badSp); }));
        bfly::Context invalid;
        CHECK(invalid.init(profile, badSp, "builtin") == -4);
    }
    CHECK(fake::streamsCreated == 0);

    // ---- runtime errors at init
    {
        fake::deviceCountValue = 0;
        bfly::Context noDevice;
        CHECK(noDevice.init(profile, space, "builtin") == -1);
        fake::deviceCountValue = 1;
        bfly::Context badDevice;
        CHECK(badDevice.init(profile, space, "builtin", 3) == -2);
    }

    bfly::Context context;
    CHECK(context.init(profile, space, "builtin") == 0);
    CHECK(fake::streamsCreated == 1);
    CHECK(context.init(profile, space, "builtin") == -9);
    CHECK(fake::streamsCreated == 1);
    CHECK(context.hardware().smCount == 148);

    // ---- candidates and lowering
    auto candidates = context.enumerate(64, 1);
    std::unique_ptr<bfly::Plan> plan;
    for (const auto& c : candidates)
        if (c.state != bfly::State::Infeasible && c.p.radix == 16 && c.a.ctaThreads == 256) {
            plan = context.makePlan(c);
            break;
        }
    CHECK(plan);
    const auto canonical = plan->candidate();
    const std::vector<std::function<void(bfly::Candidate&)>> mutations = {
        [](auto& c) { c.p.fusionLevel = 2; },
        [](auto& c) { c.p.coefficientResidency = false; },
        [](auto& c) { c.p.radix = 4; },
        [](auto& c) { c.l.contiguous = false; },
        [](auto& c) { c.l.in = bfly::Layout::Planar; },
        [](auto& c) { c.l.out = bfly::Layout::Planar; },
        [](auto& c) { c.a.level = 1; },
        [](auto& c) { c.a.ctaThreads = 0; },
        [](auto& c) { c.a.ctaThreads = 96; },
        [](auto& c) { c.a.localExchange = "shuffle"; },
        [](auto& c) { c.a.localExchange = "register"; },
        [](auto& c) { c.f.precision = "split_bf16"; },
        [](auto& c) { c.f.schedule = "bogus"; },
        [](auto& c) { c.state = bfly::State::Infeasible; }};
    for (const auto& mutate : mutations) {
        auto c = canonical;
        mutate(c);
        CHECK(!context.makePlan(c));
    }
    bfly::Context uninitialized;
    CHECK(!uninitialized.makePlan(canonical));
    {
        bfly::Context missingKernel;
        CHECK(missingKernel.init(profile, space, tmp + "/does-not-exist.so") == 0);
        CHECK(!missingKernel.makePlan(canonical));
    }
    int feasible = 0;
    for (const auto& c : candidates) {
        if (c.state != bfly::State::Infeasible) {
            CHECK(context.makePlan(c));
            ++feasible;
        }
        if (c.a.localExchange != "shared" || c.l.in != bfly::Layout::Interleaved ||
            c.l.out != bfly::Layout::Interleaved)
            CHECK(c.state == bfly::State::Infeasible && !c.reason.empty());
        if (c.f.schedule != "stockham") CHECK(c.state == bfly::State::Infeasible);   // n <= 4096
    }
    CHECK(feasible > 0);

    // infeasibility reasons carry a key
    auto reasonFor = [&](uint32_t n, uint32_t batch) {
        std::string all;
        for (const auto& c : context.enumerate(n, batch)) {
            CHECK(c.state == bfly::State::Infeasible);
            all += c.reason + "\n";
        }
        return all;
    };
    CHECK(reasonFor(16, 64).find("minimum") != std::string::npos);
    CHECK(reasonFor(72, 64).find("power of two") != std::string::npos);
    CHECK(reasonFor(192, 64).find("power of two") != std::string::npos);
    CHECK(reasonFor(131072, 1).find("envelope") != std::string::npos);
    CHECK(reasonFor(64, 0).find("batch") != std::string::npos);
    CHECK(reasonFor(4096, 524288).find("uint32") != std::string::npos);
    {   // the uint32 offset boundary of the host-pointer API: 524287 live, 524288 rejected
        bool live = false;
        for (const auto& c : context.enumerate(4096, 524287)) live = live || c.state != bfly::State::Infeasible;
        CHECK(live);
    }
    {   // long lengths: four-step, ring and cluster feasible, single CTA only up to 16384
        int fs = 0, cl = 0, rg = 0, sp = 0;
        for (const auto& c : context.enumerate(65536, 4))
            if (c.state != bfly::State::Infeasible)
                (c.f.schedule == "four_step" ? fs : c.f.schedule == "cluster" ? cl : c.f.schedule == "ring" ? rg : sp)++;
        CHECK(fs == 1 && cl == 2 && rg == 1 && sp == 0);   // cluster: 256- and 512-thread CTAs
        bool single8192 = false;
        for (const auto& c : context.enumerate(8192, 4))
            single8192 = single8192 || (c.state != bfly::State::Infeasible && c.f.schedule == "stockham");
        CHECK(single8192);
        // which kernels prepare() lowers a 65536-point C2C to, per schedule
        auto launchLabel = [&](const std::string& sched) {
            for (const auto& c : context.enumerate(65536, 4))
                if (c.state != bfly::State::Infeasible && c.f.schedule == sched) {
                    auto pl = context.makePlan(c);
                    if (!pl || pl->prepare(65536, 2) != 0) return std::string("<no plan>");
                    for (const auto& t : pl->transforms())
                        if (t.kind == bfly::Transform::LaunchKernel) return t.label;
                }
            return std::string("<none>");
        };
        CHECK(launchLabel("cluster").find("cluster") != std::string::npos);
        CHECK(launchLabel("four_step").find("four-step") != std::string::npos);
        CHECK(launchLabel("ring").find("L2 ring") != std::string::npos);
        CHECK(fake::allocations == fake::releases && fake::launches > 0);   // plans freed their tables
        fake::allocations = fake::releases = fake::copies = fake::launches = 0;
    }

    // ---- guards: -8 before any allocation, copy or launch
    float dummy[4] = {0, 0, 0, 0};
    for (uint32_t n : {0u, 1u, 32u, 192u, 16384u}) {
        CHECK(plan->run(dummy, dummy, n, 1) == -8);
        CHECK(plan->runR2C(dummy, dummy, n, 1) == -8);
        CHECK(plan->runC2R(dummy, dummy, n, 1) == -8);
    }
    for (uint32_t n : {0u, 1u, 16u, 192u, 131072u}) CHECK(plan->prepare(n, 1) == -8);
    CHECK(plan->run(dummy, dummy, 8192, 1) == -8);
    CHECK(plan->runC2R(dummy, dummy, 8192, 1) == -8);
    CHECK(plan->runR2C(dummy, dummy, 64, 1) == -8);
    CHECK(plan->runLong(dummy, dummy, 4096, 1, -1) == -8);
    CHECK(plan->runLong(dummy, dummy, 8192, 1, 0) == -8);
    for (auto run : {&bfly::Plan::run, &bfly::Plan::runR2C, &bfly::Plan::runC2R}) {
        CHECK((plan.get()->*run)(dummy, dummy, 128, 0) == -8);
        CHECK((plan.get()->*run)(nullptr, dummy, 128, 1) == -8);
        CHECK((plan.get()->*run)(dummy, nullptr, 128, 1) == -8);
        CHECK((plan.get()->*run)(dummy, dummy, 128, 0xffffffffu) == -8);
    }
    CHECK(plan->execC2C(nullptr, dummy, 64, 1, -1, 1.f, nullptr) == -8);
    CHECK(plan->execC2C(dummy, dummy, 64, 0, -1, 1.f, nullptr) == -8);
    CHECK(plan->execC2C(dummy, dummy, 64, 1, 0, 1.f, nullptr) == -8);
    CHECK(plan->execC2C(dummy, dummy, 9001, 1, -1, 1.f, nullptr) == -8);   // prime, above the Bluestein envelope
    CHECK(plan->execC2C(dummy, dummy, 12348, 1, -1, 1.f, nullptr) == -8);  // 2^2 3^2 7^3: 7-smooth, above 12288
    CHECK(plan->execC2C(dummy, dummy, 1, 1, -1, 1.f, nullptr) == -8);
    CHECK(plan->execC2C(dummy, dummy, 131072, 1, -1, 1.f, nullptr) == -8);
    CHECK(plan->execR2C(dummy, dummy, 32, 1, 1.f, 1.f, nullptr) == -8);
    CHECK(plan->execC2R(dummy, dummy, 16384, 1, 1.f, 1.f, 1.f, nullptr) == -8);
    bfly::Metric metric;
    CHECK(plan->measure(1, 1, &metric) == -8);
    CHECK(plan->measure(64, 1, nullptr) == -1);
    CHECK(plan->prepare(64, 0) == -8);
    CHECK(fake::allocations == 0 && fake::copies == 0 && fake::launches == 0);

    // ---- failure injection: a failed prepare never leaves a usable stale key
    CHECK(plan->prepare(64, 1) == 0);
    const int afterFirst = fake::allocations;
    CHECK(afterFirst == 1);
    fake::failAllocation = fake::allocations + 1;
    CHECK(plan->prepare(128, 1) != 0);
    fake::failAllocation = 0;
    int before = fake::allocations;
    CHECK(plan->prepare(128, 1) == 0);          // rebuilt, not served from a stale entry
    CHECK(fake::allocations == before + 1);
    fake::failLaunch = fake::launches + 1;      // twiddle build fails
    CHECK(plan->prepare(256, 1) != 0);
    fake::failLaunch = 0;
    before = fake::allocations;
    CHECK(plan->prepare(256, 1) == 0);
    CHECK(fake::allocations == before + 1);
    before = fake::allocations;
    CHECK(plan->prepare(64, 1) == 0);            // cached
    CHECK(plan->prepare(128, 1) == 0);
    CHECK(fake::allocations == before);

    // ---- host round trip: status code per failing step, correct values otherwise
    const uint32_t n = 64, batch = 3;
    std::vector<float> in(2 * n * batch), out(2 * n * batch), ref(2 * n);
    for (size_t i = 0; i < in.size(); ++i) in[i] = bfly::patternAt(i);
    CHECK(plan->run(in.data(), out.data(), n, batch) == 0);
    for (uint32_t b = 0; b < batch; ++b) {
        bfly::refFftF32(in.data() + b * 2 * n, ref.data(), n);
        CHECK(bfly::maxRelScaled(out.data() + b * 2 * n, ref.data(), 2 * n) < 1e-5);
    }
    fake::failCopy = fake::copies + 1;
    CHECK(plan->run(in.data(), out.data(), n, batch) == -4);
    fake::failCopy = fake::copies + 2;
    CHECK(plan->run(in.data(), out.data(), n, batch) == -7);
    fake::failCopy = 0;
    fake::failLaunch = fake::launches + 1;
    CHECK(plan->run(in.data(), out.data(), n, batch) == -5);
    fake::failLaunch = 0;
    fake::failSync = fake::syncs + 1;
    CHECK(plan->run(in.data(), out.data(), n, batch) == -6);
    fake::failSync = 0;
    fake::failAllocation = fake::allocations + 1;
    CHECK(plan->run(in.data(), out.data(), 128, 4) == -3);   // larger buffers must grow
    fake::failAllocation = 0;
    CHECK(plan->run(in.data(), out.data(), n, batch) == 0);
    CHECK(plan->runInverse(out.data(), out.data(), n, batch, 1.0f / n) == 0);
    for (size_t i = 0; i < in.size(); ++i) CHECK(std::fabs(out[i] - in[i]) < 1e-5);

    // ---- large batch: the round trip is pipelined over row chunks on three streams
    {
        const uint32_t bn = 64, bb = 17000;   // 2 x 8.7 MB > 4 MB pipelining threshold
        std::vector<float> bin(2 * (size_t)bn * bb), bout(bin.size()), bref(2 * bn);
        for (size_t i = 0; i < bin.size(); ++i) bin[i] = bfly::patternAt(i * 3 + 1);
        const int streamsBefore = fake::streamsCreated;
        CHECK(plan->run(bin.data(), bout.data(), bn, bb) == 0);
        CHECK(fake::streamsCreated == streamsBefore + 2);
        uint32_t rows[8];
        const uint32_t cnt = bfly::sampleBatches(bb, 8, rows, 8);
        for (uint32_t i = 0; i < cnt; ++i) {
            bfly::refFftF32(bin.data() + (size_t)rows[i] * 2 * bn, bref.data(), bn);
            CHECK(bfly::maxRelScaled(bout.data() + (size_t)rows[i] * 2 * bn, bref.data(), 2 * bn) < 1e-5);
        }
        fake::failCopy = fake::copies + 3;   // the second chunk's upload (4 MB chunks: 8192 rows)
        const int rc = plan->run(bin.data(), bout.data(), bn, bb);
        CHECK(rc == -4);
        fake::failCopy = 0;
    }

    // ---- measure: acceptance against the FP64 check, state transitions
    CHECK(plan->measure(64, 2, &metric) == 0);
    CHECK(metric.measuredOk && metric.maxRelErr < 1e-5 && plan->candidate().state == bfly::State::Measured);
    CHECK(std::fabs(metric.measuredUs - fake::timerMs * 1000.0) < 1e-6);

    // ---- select + tuning cache
    const std::string cache = tmp + "/tune.json";
    context.setTuningCache(cache);
    std::string log;
    auto best = context.select(64, 2, 2, &log);
    CHECK(best);
    CHECK(log.find("accept") != std::string::npos && log.find("selected:") != std::string::npos);
    CHECK(read(cache).find(best->candidate().id) != std::string::npos);
    const int launchesBefore = fake::launches;
    std::string log2;
    auto cached = context.select(64, 2, 2, &log2);
    CHECK(cached && cached->candidate().id == best->candidate().id);
    CHECK(log2.find("tuning cache") != std::string::npos);
    CHECK(fake::launches == launchesBefore);   // no measurement
    write(cache, "{ not json");
    std::string log3;
    CHECK(context.select(64, 2, 1, &log3));    // corrupt cache ignored and rewritten
    CHECK(read(cache).find("schema_version") != std::string::npos);

    // ---- ragged work list: invalid requests rejected before allocation, values correct
    {
        std::vector<float> a(2 * 64 * 3), b(2 * 128 * 2), oa(a.size()), ob(b.size()), r(2 * 128);
        for (size_t i = 0; i < a.size(); ++i) a[i] = bfly::patternAt(i);
        for (size_t i = 0; i < b.size(); ++i) b[i] = bfly::patternAt(i + 7);
        const int allocBefore = fake::allocations;
        int st = 0;
        bfly::RaggedRequest bad[] = {{a.data(), oa.data(), 96, 3, -1, 1.f}};
        CHECK(!plan->makeRagged(bad, 1, &st) && st == -8);
        bfly::RaggedRequest bad2[] = {{a.data(), oa.data(), 8192, 3, -1, 1.f}};
        CHECK(!plan->makeRagged(bad2, 1, &st) && st == -8);
        bfly::RaggedRequest bad3[] = {{a.data(), oa.data(), 64, 0, -1, 1.f}};
        CHECK(!plan->makeRagged(bad3, 1, &st) && st == -8);
        CHECK(!plan->makeRagged(nullptr, 1, &st) && st == -8);
        CHECK(fake::allocations == allocBefore);
        bfly::RaggedRequest ok[] = {{a.data(), oa.data(), 64, 3, -1, 1.f}, {b.data(), ob.data(), 128, 2, 1, 0.5f}};
        auto rg = plan->makeRagged(ok, 2, &st);
        CHECK(rg && st == 0 && rg->requests() == 2);
        CHECK(rg->tiles() == 1 + 1);   // 64-point: 32 rows per tile; 128-point: 32 rows per tile
        CHECK(rg->exec(nullptr) == 0);
        for (uint32_t row = 0; row < 3; ++row) {
            bfly::refFftF32(a.data() + row * 128, r.data(), 64);
            CHECK(bfly::maxRelScaled(oa.data() + row * 128, r.data(), 128) < 1e-5);
        }
        fake::failAllocation = fake::allocations + 1;
        CHECK(!plan->makeRagged(ok, 2, &st) && st == -3);
        fake::failAllocation = 0;

        // explicit configurations: the radix sets the rows per tile, invalid ones are refused
        std::vector<float> c(2 * 128 * 20), oc(c.size());
        for (size_t i = 0; i < c.size(); ++i) c[i] = bfly::patternAt(i + 11);
        bfly::RaggedRequest mix[] = {{a.data(), oa.data(), 64, 3, -1, 1.f}, {c.data(), oc.data(), 128, 20, -1, 1.f}};
        bfly::RaggedConfig all8{-1, 0x7F}, all16{-1, 0x0};
        auto r8 = plan->makeRagged(mix, 2, &st, &all8);
        CHECK(r8 && st == 0 && r8->tiles() == 1 + 2);   // 64: 32 rows per tile; 128: 16 rows per tile
        CHECK(r8->config().radix8 == 0x7F && r8->config().mode == -1);
        CHECK(r8->exec(nullptr) == 0);
        bfly::refFftF32(c.data() + 19 * 256, r.data(), 128);
        CHECK(bfly::maxRelScaled(oc.data() + 19 * 256, r.data(), 256) < 1e-5);
        auto r16 = plan->makeRagged(mix, 2, &st, &all16);
        CHECK(r16 && r16->tiles() == 1 + 1);            // 64: 64 rows per tile; 128: 32 rows per tile
        const int allocBad = fake::allocations;
        bfly::RaggedConfig bad4096{-1, 0x80}, badMode{3, 0x3}, staged{1, 0x3};
        CHECK(!plan->makeRagged(mix, 2, &st, &bad4096) && st == -8);
        CHECK(!plan->makeRagged(mix, 2, &st, &badMode) && st == -8);
        bfly::RaggedRequest odd[] = {{c.data() + 2, oc.data(), 64, 1, -1, 1.f}};   // 8-byte aligned input
        CHECK(!plan->makeRagged(odd, 1, &st, &staged) && st == -8);
        CHECK(fake::allocations == allocBad);
        auto rs = plan->makeRagged(mix, 2, &st, &staged);
        CHECK(rs && rs->stages() == 1 && rs->aligned());

        // autotuner: 16-value tiles made slower by the fake timer, so both lengths present move
        // to 8 values; the modes cost the same and stay at the default; the choice is persisted
        // and reused without measuring
        fake::raggedCost16 = 4;
        std::string tlog;
        auto tuned = context.tuneRagged(*plan, ok, 2, &st, &tlog);
        CHECK(tuned && st == 0);
        CHECK(tuned->config().radix8 == 0x7 && tuned->config().mode == -1);
        CHECK(tlog.find("selected: mode -1 radix8 0x07") != std::string::npos);
        CHECK(read(cache).find("\"kind\": \"ragged\"") != std::string::npos);
        const int launchesTuned = fake::launches;
        std::string tlog2;
        auto again = context.tuneRagged(*plan, ok, 2, &st, &tlog2);
        CHECK(again && again->config().radix8 == 0x7 && tlog2.find("tuning cache") != std::string::npos);
        CHECK(fake::launches == launchesTuned);
        bfly::RaggedRequest other[] = {{a.data(), oa.data(), 64, 2, -1, 1.f}};   // another shape: measured
        auto t3 = context.tuneRagged(*plan, other, 1, &st, nullptr);
        CHECK(t3 && t3->config().radix8 == 0x3 && fake::launches > launchesTuned);
        CHECK(!context.tuneRagged(*plan, bad, 1, &st, nullptr) && st == -8);
        fake::raggedCost16 = 0;
    }

    {   // 2-D and middle-axis transforms: exact against a direct FP64 DFT of the same layout
        auto dft2 = [](const std::vector<float>& x, uint32_t ny, uint32_t nx, uint32_t batch, int sign) {
            std::vector<double> y(x.size());
            for (uint32_t b = 0; b < batch; ++b)
                for (uint32_t ky = 0; ky < ny; ++ky)
                    for (uint32_t kx = 0; kx < nx; ++kx) {
                        double re = 0, im = 0;
                        for (uint32_t iy = 0; iy < ny; ++iy)
                            for (uint32_t ix = 0; ix < nx; ++ix) {
                                const double a = sign * 2 * M_PI *
                                                 ((double)((iy * ky) % ny) / ny + (double)((ix * kx) % nx) / nx);
                                const size_t at = 2 * (((size_t)b * ny + iy) * nx + ix);
                                re += x[at] * std::cos(a) - x[at + 1] * std::sin(a);
                                im += x[at] * std::sin(a) + x[at + 1] * std::cos(a);
                            }
                        const size_t o = 2 * (((size_t)b * ny + ky) * nx + kx);
                        y[o] = re;
                        y[o + 1] = im;
                    }
            return y;
        };
        auto maxErr = [](const std::vector<float>& got, const std::vector<double>& ref, double scale) {
            double e = 0, m = 0;
            for (size_t i = 0; i < got.size(); ++i) {
                e = std::max(e, std::fabs(got[i] - ref[i] * scale));
                m = std::max(m, std::fabs(ref[i] * scale));
            }
            return e / std::max(1.0, m);
        };
        const uint32_t ny = 32, nx = 64, batch = 2;
        std::vector<float> x(2 * ny * nx * batch), y(x.size());
        for (size_t i = 0; i < x.size(); ++i) x[i] = (float)std::sin(0.37 * i + 0.1 * (i % 7));
        CHECK(plan->execC2C2D(x.data(), y.data(), ny, nx, batch, -1, 1.f, nullptr) == 0);
        CHECK(maxErr(y, dft2(x, ny, nx, batch, -1), 1.0) < 1e-5);
        CHECK(plan->execC2C2D(x.data(), y.data(), ny, nx, batch, 1, 0.25f, nullptr) == 0);
        CHECK(maxErr(y, dft2(x, ny, nx, batch, 1), 0.25) < 1e-5);
        // middle axis of [outer][n][inner]: the same data read as [2][32][64] transformed along
        // the 32-point axis equals the column pass of the 2-D transform alone
        std::vector<float> axis(x.size());
        CHECK(plan->execC2CAxis(x.data(), axis.data(), 32, 2, 64, -1, 1.f, nullptr) == 0);
        double e = 0;
        for (uint32_t b = 0; b < 2; ++b)
            for (uint32_t c = 0; c < 64; ++c)
                for (uint32_t k = 0; k < 32; ++k) {
                    double re = 0, im = 0;
                    for (uint32_t i = 0; i < 32; ++i) {
                        const double a = -2 * M_PI * (double)((i * k) % 32) / 32;
                        const size_t at = 2 * (((size_t)b * 32 + i) * 64 + c);
                        re += x[at] * std::cos(a) - x[at + 1] * std::sin(a);
                        im += x[at] * std::sin(a) + x[at + 1] * std::cos(a);
                    }
                    const size_t o = 2 * (((size_t)b * 32 + k) * 64 + c);
                    e = std::max(e, std::max(std::fabs(axis[o] - re), std::fabs(axis[o + 1] - im)));
                }
        CHECK(e < 1e-3);
        // in place, and inner == 1 is the plain row transform
        std::vector<float> inplace = x;
        CHECK(plan->execC2CAxis(inplace.data(), inplace.data(), 32, 2, 64, -1, 1.f, nullptr) == 0);
        CHECK(inplace == axis);
        std::vector<float> rows1(x.size()), rows2(x.size());
        CHECK(plan->execC2CAxis(x.data(), rows1.data(), 64, 64, 1, -1, 1.f, nullptr) == 0);
        CHECK(plan->execC2C(x.data(), rows2.data(), 64, 64, -1, 1.f, nullptr) == 0);
        CHECK(rows1 == rows2);
        // guards: -8 before any allocation or launch
        const int allocBefore = fake::allocations, launchBefore = fake::launches;
        float* d = x.data();
        CHECK(plan->execC2C2D(nullptr, d, 32, 64, 1, -1, 1.f, nullptr) == -8);
        CHECK(plan->execC2C2D(d, d, 32, 64, 0, -1, 1.f, nullptr) == -8);
        CHECK(plan->execC2C2D(d, d, 32, 64, 1, 2, 1.f, nullptr) == -8);
        CHECK(plan->execC2C2D(d, d, 16, 64, 1, -1, 1.f, nullptr) == -8);      // ny below 32
        CHECK(plan->execC2C2D(d, d, 8192, 64, 1, -1, 1.f, nullptr) == -8);    // ny above 4096
        CHECK(plan->execC2C2D(d, d, 48, 64, 1, -1, 1.f, nullptr) == -8);      // ny not a power of two
        CHECK(plan->execC2C2D(d, d, 32, 9001, 1, -1, 1.f, nullptr) == -8);    // nx beyond every row kernel
        CHECK(plan->execC2C2D(d, d, 4096, 64, 1u << 20, -1, 1.f, nullptr) == -8);   // batch*ny > 2^32-1
        // batch * ny wraps to a small value in 64 bits (2^52 * 4096 = 2^64 -> 0; +1 row -> 4096)
        CHECK(plan->execC2C2D(d, d, 4096, 64, (1ull << 52) + 1, -1, 1.f, nullptr) == -8);
        CHECK(plan->execR2C2D(d, d, 4096, 64, (1ull << 52) + 1, 1.f, nullptr) == -8);
        CHECK(plan->execC2R2D(d, d, 4096, 64, (1ull << 52) + 1, 1.f, nullptr) == -8);
        CHECK(plan->execC2CAxis(d, d, 32, 0, 3, -1, 1.f, nullptr) == -8);
        CHECK(plan->execC2CAxis(d, d, 32, 1, 0, -1, 1.f, nullptr) == -8);
        CHECK(plan->execC2CAxis(d, d, 8192, 1, 3, -1, 1.f, nullptr) == -8);   // strided n above 4096
        CHECK(plan->execC2CAxis(d, d, 100, 1, 3, -1, 1.f, nullptr) == -8);
        CHECK(plan->execR2C2D(nullptr, d, 32, 64, 1, 1.f, nullptr) == -8);
        CHECK(plan->execR2C2D(d, d, 48, 64, 1, 1.f, nullptr) == -8);        // ny not a power of two
        CHECK(plan->execR2C2D(d, d, 32, 34, 1, 1.f, nullptr) == -8);        // nx outside R2C (17 is not 13-smooth)
        CHECK(plan->execC2R2D(d, d, 8192, 64, 1, 1.f, nullptr) == -8);      // ny above 4096
        CHECK(plan->execC2R2D(d, d, 32, 16384, 1, 1.f, nullptr) == -8);     // nx outside C2R
        CHECK(plan->execC2R2D(d, d, 32, 64, 0, 1.f, nullptr) == -8);
        CHECK(fake::allocations == allocBefore && fake::launches == launchBefore);
    }

    {   // STFT: frame count, centred reflect padding and window against a direct DFT
        const uint32_t n = 64, hop = 24;
        const uint64_t len = 200, signals = 2;
        std::vector<float> sig(len * signals), win(n);
        for (size_t i = 0; i < sig.size(); ++i) sig[i] = (float)std::cos(0.05 * i * i / 7.0 + i % 3);
        for (uint32_t j = 0; j < n; ++j) win[j] = (float)(0.5 - 0.5 * std::cos(2 * M_PI * j / n));
        for (bool center : {true, false}) {
            const uint64_t frames = center ? 1 + len / hop : 1 + (len - n) / hop;
            std::vector<float> spec(2 * (n / 2 + 1) * frames * signals);
            uint64_t got = 0;
            CHECK(plan->execStft(sig.data(), spec.data(), n, signals, len, hop, center, win.data(), &got, nullptr) == 0);
            CHECK(got == frames);
            double e = 0;
            for (uint64_t s2 = 0; s2 < signals; ++s2)
                for (uint64_t f = 0; f < frames; ++f)
                    for (uint32_t k = 0; k <= n / 2; ++k) {
                        double re = 0, im = 0;
                        for (uint32_t j = 0; j < n; ++j) {
                            long long i = (long long)(f * hop + j) - (center ? n / 2 : 0);
                            if (i < 0) i = -i;
                            if (i >= (long long)len) i = 2 * ((long long)len - 1) - i;
                            const double v = sig[s2 * len + i] * win[j];
                            const double a = -2 * M_PI * (double)((j * k) % n) / n;
                            re += v * std::cos(a);
                            im += v * std::sin(a);
                        }
                        const size_t o = 2 * ((s2 * frames + f) * (n / 2 + 1) + k);
                        e = std::max(e, std::max(std::fabs(spec[o] - re), std::fabs(spec[o + 1] - im)));
                    }
            CHECK(e < 1e-3);
        }
        const int allocBefore = fake::allocations, launchBefore = fake::launches;
        float* d = sig.data();
        uint64_t fr = 0;
        CHECK(plan->execStft(nullptr, d, 64, 1, 200, 16, true, nullptr, &fr, nullptr) == -8);
        CHECK(plan->execStft(d, d, 34, 1, 200, 16, true, nullptr, &fr, nullptr) == -8);     // 17 is not 13-smooth
        CHECK(plan->execStft(d, d, 32, 1, 200, 16, true, nullptr, &fr, nullptr) == -8);     // below 64
        CHECK(plan->execStft(d, d, 16384, 1, 20000, 16, true, nullptr, &fr, nullptr) == -8);
        CHECK(plan->execStft(d, d, 64, 1, 200, 0, true, nullptr, &fr, nullptr) == -8);      // hop 0
        CHECK(plan->execStft(d, d, 64, 0, 200, 16, true, nullptr, &fr, nullptr) == -8);     // no signals
        CHECK(plan->execStft(d, d, 64, 1, 32, 16, true, nullptr, &fr, nullptr) == -8);      // reflect needs len > n/2
        CHECK(plan->execStft(d, d, 64, 1, 63, 16, false, nullptr, &fr, nullptr) == -8);     // shorter than a frame
        CHECK(plan->execStft(d, d, 64, 1, 200, 16, true, d + 1, &fr, nullptr) == -8);       // window not 8-byte aligned
        CHECK(fake::allocations == allocBefore && fake::launches == launchBefore);
    }

    {   // mixed-radix planner: every 13-smooth n up to kMixedMaxN (and no other) gets a plan of
        // radices the kernel implements whose product is n, with consistent Ns and twiddle offsets
        int plans = 0, maxPasses = 0;
        for (uint32_t n = 2; n <= bfly::backend::kMixedMaxN; ++n) {
            uint32_t r = n;
            for (uint32_t p : {2u, 3u, 5u, 7u, 11u, 13u})
                while (r % p == 0) r /= p;
            bfly::backend::MixedRadix m;
            const bool ok = bfly::backend::mixedRadix(n, &m);
            CHECK(ok == (r == 1));
            if (!ok) continue;
            ++plans;
            maxPasses = std::max(maxPasses, m.passes);
            uint64_t prod = 1;
            int tw = 0;
            for (int q = 0; q < m.passes; ++q) {
                const int R = m.radix[q];
                CHECK(R == 2 || R == 3 || R == 4 || R == 5 || R == 6 || R == 7 || R == 8 || R == 9 || R == 10 ||
                      R == 11 || R == 12 || R == 13 || R == 14 || R == 15 || R == 16);
                CHECK(m.ns[q] == (int)prod && m.twoff[q] == tw);
                if (q) tw += (R - 1) * m.ns[q];
                prod *= (uint64_t)R;
            }
            CHECK(prod == n && m.twsize == tw && m.n == (int)n);
        }
        CHECK(plans == 799 && maxPasses <= 5);
        bfly::backend::MixedRadix m;
        CHECK(bfly::backend::mixedRadix(1000, &m) && m.passes == 3 && m.radix[0] == 10);      // 10^3
        CHECK(bfly::backend::mixedRadix(10000, &m) && m.passes == 4);                           // 10^4, not 16 5^4
        CHECK(bfly::backend::mixedRadix(6561, &m) && m.passes == 4 && m.radix[0] == 9);        // 9^4
        CHECK(!bfly::backend::mixedRadix(12348, nullptr) && !bfly::backend::mixedRadix(17, nullptr));
    }

    {   // real transforms of even non-power-of-two n (n/2 13-smooth): R2C matches a direct DFT,
        // C2R (1/n) brings the signal back, each one launch once the tables exist
        const uint32_t n = 96;
        const uint64_t batch = 3;
        std::vector<float> x(n * batch), back(n * batch), spec(2 * (n / 2 + 1) * batch);
        for (size_t i = 0; i < x.size(); ++i) x[i] = (float)std::sin(0.37 * i + std::cos(0.11 * i));
        CHECK(plan->execR2C(x.data(), spec.data(), n, batch, 1.f, 1.f, nullptr) == 0);
        const int l0 = fake::launches;
        CHECK(plan->execR2C(x.data(), spec.data(), n, batch, 1.f, 1.f, nullptr) == 0);
        CHECK(fake::launches == l0 + 1);
        double e = 0;
        for (uint64_t b = 0; b < batch; ++b)
            for (uint32_t k = 0; k <= n / 2; ++k) {
                double re = 0, im = 0;
                for (uint32_t j = 0; j < n; ++j) {
                    const double a = -2 * M_PI * (double)((j * k) % n) / n;
                    re += x[b * n + j] * std::cos(a);
                    im += x[b * n + j] * std::sin(a);
                }
                const size_t o = 2 * (b * (n / 2 + 1) + k);
                e = std::max(e, std::max(std::fabs(spec[o] - re), std::fabs(spec[o + 1] - im)));
            }
        CHECK(e < 1e-3);
        CHECK(plan->execC2R(spec.data(), back.data(), n, batch, 1.f, 1.f, 1.f / n, nullptr) == 0);
        e = 0;
        for (size_t i = 0; i < x.size(); ++i) e = std::max(e, (double)std::fabs(back[i] - x[i]));
        CHECK(e < 1e-4);
        // STFT then inverse STFT of the same even non-power-of-two length gives the signal back
        {
            const uint32_t hop = 24;
            const uint64_t len = 400, frames = 1 + len / hop;
            std::vector<float> sig(len), win(n), sp(2 * (n / 2 + 1) * frames), rec(len);
            for (uint64_t i = 0; i < len; ++i) sig[i] = (float)std::sin(0.05 * i * i / 9.0);
            for (uint32_t j = 0; j < n; ++j) win[j] = (float)(0.5 - 0.5 * std::cos(2 * M_PI * j / n)) + 0.1f;
            uint64_t got = 0;
            CHECK(plan->execStft(sig.data(), sp.data(), n, 1, len, hop, true, win.data(), &got, nullptr) == 0);
            CHECK(got == frames);
            CHECK(plan->execIstft(sp.data(), rec.data(), n, 1, (uint32_t)frames, hop, true, win.data(), len, 1.f,
                                  nullptr) == 0);
            double er = 0;
            for (uint64_t i = 0; i < len; ++i) er = std::max(er, (double)std::fabs(rec[i] - sig[i]));
            CHECK(er < 1e-4);
        }
        CHECK(plan->execR2C(x.data(), spec.data(), 34, batch, 1.f, 1.f, nullptr) == -8);   // 17 is not 13-smooth
        CHECK(plan->execC2R(spec.data(), back.data(), 97, batch, 1.f, 1.f, 1.f, nullptr) == -8);   // odd
    }

    {   // inverse STFT: STFT then ISTFT gives the signal back (Hann window, centred, hop n/4),
        // one launch, no allocation once the real-transform tables exist; guards first
        const uint32_t n = 64, hop = 16;
        const uint64_t len = 256, signals = 2, frames = 1 + len / hop;
        std::vector<float> sig(len * signals), win(n), back(len * signals, -1.f);
        std::vector<float> spec(2 * (n / 2 + 1) * frames * signals);
        for (size_t i = 0; i < sig.size(); ++i) sig[i] = (float)std::sin(0.11 * i + std::cos(0.03 * i));
        for (uint32_t j = 0; j < n; ++j) win[j] = (float)(0.5 - 0.5 * std::cos(2 * M_PI * j / n));
        float* d = sig.data();
        const int allocBefore = fake::allocations, launchBefore = fake::launches;
        CHECK(plan->execIstft(nullptr, d, n, 1, frames, hop, true, nullptr, len, 1.f, nullptr) == -8);
        CHECK(plan->execIstft(d, d, 34, 1, frames, hop, true, nullptr, len, 1.f, nullptr) == -8);   // 17 is not 13-smooth
        CHECK(plan->execIstft(d, d, n, 1, frames, 0, true, nullptr, len, 1.f, nullptr) == -8);     // hop 0
        CHECK(plan->execIstft(d, d, n, 1, frames, n + 1, true, nullptr, len, 1.f, nullptr) == -8); // hop above n
        // signals * frames wraps to a small value in 64 bits: still too many rows
        CHECK(plan->execIstft(d, d, n, (1ull << 63) + 1, 2, hop, true, nullptr, len, 1.f, nullptr) == -8);
        CHECK(plan->execIstftBackward(d, d, n, (1ull << 63) + 1, 2, hop, true, nullptr, len, 1.f, nullptr) == -8);
        CHECK(plan->execStftBackward(d, d, n, (1ull << 62) + 1, 4 * (uint64_t)hop, hop, false, nullptr, nullptr) == -8);
        CHECK(plan->execStftBackward(d, d, n, 1, n + 1, hop, true, nullptr, nullptr) == -8);   // centred: n + 2 samples
        CHECK(plan->execIstft(d, d, n, 0, frames, hop, true, nullptr, len, 1.f, nullptr) == -8);   // no signals
        CHECK(plan->execIstft(d, d, n, 1, 0, hop, true, nullptr, len, 1.f, nullptr) == -8);        // no frames
        CHECK(plan->execIstft(d, d, n, 1, frames, hop, true, nullptr, 0, 1.f, nullptr) == -8);     // empty output
        CHECK(fake::allocations == allocBefore && fake::launches == launchBefore);
        uint64_t got = 0;
        CHECK(plan->execStft(sig.data(), spec.data(), n, signals, len, hop, true, win.data(), &got, nullptr) == 0);
        CHECK(got == frames);
        for (int rep = 0; rep < 2; ++rep) {
            const int a0 = fake::allocations, l0 = fake::launches;
            CHECK(plan->execIstft(spec.data(), back.data(), n, signals, (uint32_t)frames, hop, true, win.data(), len,
                                  1.f, nullptr) == 0);
            CHECK(fake::launches == l0 + 1);
            CHECK(fake::allocations == a0);
        }
        double e = 0;
        for (size_t i = 0; i < sig.size(); ++i) e = std::max(e, (double)std::fabs(back[i] - sig[i]));
        CHECK(e < 1e-4);
        // uncentred, rectangular window, scale 2: frames cover [0, n + (frames-1) hop) exactly
        const uint64_t fr2 = 1 + (len - n) / hop, out2 = n + (fr2 - 1) * hop;
        CHECK(plan->execStft(sig.data(), spec.data(), n, 1, len, hop, false, nullptr, &got, nullptr) == 0);
        CHECK(got == fr2);
        CHECK(plan->execIstft(spec.data(), back.data(), n, 1, (uint32_t)fr2, hop, false, nullptr, out2 + 5, 2.f,
                              nullptr) == 0);
        e = 0;
        for (uint64_t i = 0; i < out2; ++i) e = std::max(e, (double)std::fabs(back[i] - 2 * sig[i]));
        for (uint64_t i = out2; i < out2 + 5; ++i) e = std::max(e, (double)std::fabs(back[i]));   // past the frames: 0
        CHECK(e < 1e-4);
    }

    {   // batched host round trip: equal to per-request device transforms; guards first
        std::vector<float> a(2 * 64 * 3), b(2 * 96 * 2), c(2 * 128 * 4);
        for (size_t i = 0; i < a.size(); ++i) a[i] = (float)std::sin(0.3 * i);
        for (size_t i = 0; i < b.size(); ++i) b[i] = (float)std::cos(0.7 * i + 1);
        for (size_t i = 0; i < c.size(); ++i) c[i] = (float)std::sin(1.1 * i * i);
        std::vector<float> oa(a.size()), ob(b.size()), oc(c.size()), ra(a.size()), rb(b.size()), rc2(c.size());
        const bfly::HostRequest reqs[] = {{a.data(), oa.data(), 64, 3, -1, 1.f},
                                          {b.data(), ob.data(), 96, 2, -1, 1.f},
                                          {c.data(), oc.data(), 128, 4, 1, 0.125f}};
        CHECK(plan->runMany(reqs, 3) == 0);
        CHECK(plan->execC2C(a.data(), ra.data(), 64, 3, -1, 1.f, nullptr) == 0);
        CHECK(plan->execC2C(b.data(), rb.data(), 96, 2, -1, 1.f, nullptr) == 0);
        CHECK(plan->execC2C(c.data(), rc2.data(), 128, 4, 1, 0.125f, nullptr) == 0);
        CHECK(oa == ra && ob == rb && oc == rc2);
        const int allocBefore = fake::allocations, copiesBefore = fake::copies, launchBefore = fake::launches;
        CHECK(plan->runMany(nullptr, 1) == -8);
        CHECK(plan->runMany(reqs, 0) == -8);
        const bfly::HostRequest bad1[] = {reqs[0], {a.data(), oa.data(), 9001, 1, -1, 1.f}};
        const bfly::HostRequest bad2[] = {reqs[0], {a.data(), oa.data(), 64, 1, 0, 1.f}};
        const bfly::HostRequest bad3[] = {reqs[0], {nullptr, oa.data(), 64, 1, -1, 1.f}};
        const bfly::HostRequest bad4[] = {reqs[0], {a.data(), oa.data(), 64, 0, -1, 1.f}};
        for (const auto* bad : {bad1, bad2, bad3, bad4}) CHECK(plan->runMany(bad, 2) == -8);
        CHECK(fake::allocations == allocBefore && fake::copies == copiesBefore && fake::launches == launchBefore);
    }

    {   // batched host round trip issue order: every request under 1 MB is uploaded before any
        // byte of a larger one, whatever the order the caller lists them in
        std::vector<float> big(2 * 1024 * 160), s1(2 * 64 * 3), s2(2 * 128 * 5);   // 1.25 MB, 1.5 KB, 5 KB
        for (size_t i = 0; i < big.size(); ++i) big[i] = (float)std::sin(0.01 * i);
        for (size_t i = 0; i < s1.size(); ++i) s1[i] = (float)std::cos(0.3 * i);
        for (size_t i = 0; i < s2.size(); ++i) s2[i] = (float)std::sin(0.7 * i + 2);
        std::vector<float> ob(big.size()), o1(s1.size()), o2(s2.size()), rb(big.size()), r1(s1.size()), r2(s2.size());
        const bfly::HostRequest reqs[] = {{big.data(), ob.data(), 1024, 160, -1, 1.f},
                                          {s1.data(), o1.data(), 64, 3, -1, 1.f},
                                          {s2.data(), o2.data(), 128, 5, 1, 0.5f}};
        fake::h2dSources.clear();
        CHECK(plan->runMany(reqs, 3) == 0);
        auto inside = [](const void* p, const std::vector<float>& v) {
            return p >= (const void*)v.data() && p < (const void*)(v.data() + v.size());
        };
        size_t firstBig = fake::h2dSources.size(), lastSmall = 0, smallSeen = 0;
        for (size_t i = 0; i < fake::h2dSources.size(); ++i) {
            const void* p = fake::h2dSources[i];
            if (inside(p, big)) firstBig = std::min(firstBig, i);
            if (inside(p, s1) || inside(p, s2)) { lastSmall = i; ++smallSeen; }
        }
        CHECK(smallSeen == 2 && firstBig < fake::h2dSources.size() && lastSmall < firstBig);
        CHECK(plan->execC2C(big.data(), rb.data(), 1024, 160, -1, 1.f, nullptr) == 0);
        CHECK(plan->execC2C(s1.data(), r1.data(), 64, 3, -1, 1.f, nullptr) == 0);
        CHECK(plan->execC2C(s2.data(), r2.data(), 128, 5, 1, 0.5f, nullptr) == 0);
        CHECK(ob == rb && o1 == r1 && o2 == r2);
    }

    {   // pageable host buffers go through pinned staging slots: same results as the direct path
        const uint32_t n = 64, batch = 20000;   // 10 MB each way: five pipeline chunks
        std::vector<float> x(2 * (size_t)n * batch), yDirect(x.size()), yStaged(x.size());
        for (size_t i = 0; i < x.size(); ++i) x[i] = (float)std::sin(0.001 * i + (i % 5));
        CHECK(plan->run(x.data(), yDirect.data(), n, batch) == 0);
        fake::pageableHost = true;
        CHECK(plan->run(x.data(), yStaged.data(), n, batch) == 0);
        CHECK(yStaged == yDirect);
        fake::failCopy = fake::copies + 3;          // a later upload fails
        CHECK(plan->run(x.data(), yStaged.data(), n, batch) == -4);
        fake::failCopy = 0;
        CHECK(plan->run(x.data(), yStaged.data(), n, batch) == 0);   // the plan stays usable
        CHECK(yStaged == yDirect);
        fake::pageableHost = false;
    }

    plan.reset();
    best.reset();
    cached.reset();
    CHECK(fake::releases > 0);
    std::printf("host runtime guards: all checks passed (%d allocations, %d launches)\n",
                fake::allocations, fake::launches);
    return 0;
}
