// The reference-side EPlace adapter a maintainer adds to superPlace to run its global-placement
// stages on this repository's engine (the binding INTEGRATION.md gives), compiled here against
// the reference's own headers: sp::EPlace (src/gp/eplace.h:56-77) defined over the C ABI in
// place of src/gp/eplace.cpp. Construction binds the PlaceDB, Config and MetricsSink as the
// reference's does; run(stage) uploads the PlaceDB as it is then, runs the stage as one device
// loop (spg_stage_run), writes the delivered positions back into the PlaceDB, pushes the
// stage's metrics rows into the sink and sets its summary keys (eplace.cpp:260-296, 474-517).
//
// Test infrastructure: oracle/Makefile links it with the reference's sources minus eplace.cpp
// and with the reference's own test program test/test_eplace.cpp, unmodified, so the
// reference's mGP regression checks (density sign, sanity, the already-converged no-op, the
// stagnation guard and its rollback point, determinism, the schedule diagnostics, the cGP
// macro freeze, the quality band) run against the device engine.
//
// Differences from the CPU engine, by design of the device loop:
//   * the per-iteration callback (setIterCallback) runs at every iteration with the PlaceDB's
//     positions at that iteration's evaluation point, through the engine's iteration callback
//     (each call pauses the device loop); the sink receives the stage's metrics rows when the
//     stage ends, so a callback does not see them in the sink yet;
//   * of the diagnostic GpRunOptions only freezeLambda and freezeGamma are supported; the
//     others (noMomentum, stepScale, adaptiveRestart, gradientRestart) throw.
#include <algorithm>
#include <cmath>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "db/place_db.h"
#include "gp/eplace.h"
#include "spgpu.h"
#include "util/config.h"
#include "util/invariant.h"
#include "util/metrics.h"

namespace sp {

const char* toString(GpStage s) {
    switch (s) {
        case GpStage::kMGP: return "mGP";
        case GpStage::kFillerOnly: return "FILLERONLY";
        case GpStage::kCGP: return "cGP";
    }
    return "?";
}

namespace {

void check(int rc) {
    if (rc == SPG_OK) return;
    const std::string msg = spg_last_error();
    // negative statuses map onto the reference's InvariantError kinds (src/util/invariant.h:10-19)
    if (rc == SPG_E_NON_FINITE) throw InvariantError("non_finite", "GP/device", msg);
    if (rc == SPG_E_OUT_OF_CORE) throw InvariantError("out_of_core", "GP/device", msg);
    if (rc == SPG_E_CONVERGENCE) throw InvariantError("convergence_mismatch", "GP/device", msg);
    if (rc == SPG_E_ROLLBACK) throw InvariantError("rollback_mismatch", "GP/device", msg);
    throw std::runtime_error("sm100a EPlace: " + msg);
}

spg_params params_of(const Config& cfg, const GpRunOptions& o) {
    spg_params p;
    spg_params_default(&p);
    p.target_density = cfg.target_density;
    p.target_overflow = cfg.target_overflow;
    p.cgp_target_overflow = cfg.cgp_target_overflow;
    p.gp_max_iter = cfg.gp_max_iter;
    p.ignore_net_degree = cfg.ignore_net_degree;
    p.gp_bin_dim = cfg.gp_bin_dim;
    p.filler_only_iters = cfg.filler_only_iters;
    p.delta_hpwl_ref = cfg.delta_hpwl_ref;
    p.lambda_schedule_relative = cfg.lambda_schedule == "relative";
    p.delta_hpwl_relative = cfg.delta_hpwl_relative;
    p.use_bb = cfg.use_bb;
    p.gp_backtrack = cfg.gp_backtrack;
    p.gp_stagnation_window = cfg.gp_stagnation_window;
    p.gp_stagnation_min_gain = cfg.gp_stagnation_min_gain;
    p.random_seed = cfg.random_seed;
    p.verbose = cfg.verbose;
    p.freeze_lambda = o.freezeLambda;
    p.freeze_gamma = o.freezeGamma;
    return p;
}

}  // namespace

struct EPlace::Impl {
    PlaceDB& db;
    const Config& cfg;
    MetricsSink& sink;
    IterCallback onIter;
    Impl(PlaceDB& d, const Config& c, MetricsSink& s) : db(d), cfg(c), sink(s) {}
};

EPlace::EPlace(PlaceDB& db, const Config& cfg, MetricsSink& sink) : impl_(std::make_unique<Impl>(db, cfg, sink)) {
    checkGeometry(db, "GP/initialize", false);
    check(spg_device_check());
}

EPlace::~EPlace() = default;

void EPlace::setIterCallback(IterCallback cb) { impl_->onIter = std::move(cb); }

GpResult EPlace::run(GpStage stage, GpRunOptions options) {
    Impl& s = *impl_;
    PlaceDB& db = s.db;
    if (options.noMomentum || options.stepScale != 1.f || options.adaptiveRestart || options.gradientRestart)
        throw std::runtime_error("sm100a EPlace: only the freezeLambda / freezeGamma run options are supported");
    checkGeometry(db, toString(stage), false);
    // the PlaceDB as it is now (positions, flags, fillers), rows and core as computeRegions left them
    std::vector<float> ly, rh, lx, st;
    std::vector<int32_t> ns;
    for (const auto& r : db.rows) {
        ly.push_back(r.ly);
        rh.push_back(r.height);
        lx.push_back(r.lx);
        st.push_back(r.step);
        ns.push_back(r.numSites);
    }
    spg_db_view v{};
    v.num_movable = db.numMovable;
    v.num_nodes = db.numNodes;
    v.num_fillers = db.numFillers;
    v.node_x = db.node_x.data();
    v.node_y = db.node_y.data();
    v.node_w = db.node_w.data();
    v.node_h = db.node_h.data();
    v.node_flags = db.node_flags.data();
    v.num_pins = db.numPins;
    v.pin_offset_x = db.pin_offset_x.data();
    v.pin_offset_y = db.pin_offset_y.data();
    v.pin2node = db.pin2node.data();
    v.pin2net = db.pin2net.data();
    v.num_nets = db.numNets;
    v.net2pin_start = db.net2pin_start.data();
    v.flat_net2pin = db.flat_net2pin.data();
    v.node2pin_start = db.node2pin_start.data();
    v.flat_node2pin = db.flat_node2pin.data();
    v.num_rows = static_cast<int32_t>(db.rows.size());
    v.row_ly = ly.data();
    v.row_height = rh.data();
    v.row_lx = lx.data();
    v.row_step = st.data();
    v.row_num_sites = ns.data();
    v.core_lx = db.coreRegion.lx;
    v.core_ly = db.coreRegion.ly;
    v.core_hx = db.coreRegion.hx;
    v.core_hy = db.coreRegion.hy;
    v.row_height_mode = db.rowHeight;
    v.total_row_area = db.totalRowArea;
    const spg_params p = params_of(s.cfg, options);
    spg_ctx* ctx = nullptr;
    check(spg_ctx_create(&v, &p, &ctx));
    std::unique_ptr<spg_ctx, int (*)(spg_ctx*)> guard(ctx, spg_ctx_destroy);
    // the iteration callback: the evaluation point's positions written into the PlaceDB
    struct Hook {
        Impl* s;
        GpStage stage;
    } hook{&s, stage};
    if (s.onIter) {
        spg_iter_fn fn = [](void* user, int32_t, int32_t iter, const float* x, const float* y) {
            Hook& h = *static_cast<Hook*>(user);
            PlaceDB& d = h.s->db;
            std::copy(x, x + d.totalNodes(), d.node_x.begin());
            std::copy(y, y + d.totalNodes(), d.node_y.begin());
            h.s->onIter(h.stage, iter, d);
        };
        check(spg_set_iter_callback(ctx, fn, &hook, 1));
    }
    spg_result r{};
    check(spg_stage_run(ctx, static_cast<int>(stage), &r));
    check(spg_positions_d2h(ctx, db.node_x.data(), db.node_y.data()));
    const std::string prefix = std::string(toString(stage)) + "_";
    s.sink.setSummary(prefix + "initial_hpwl", r.initial_hpwl);
    s.sink.setSummary(prefix + "initial_overflow", r.initial_overflow);
    s.sink.setSummary(prefix + "initial_lambda", r.initial_lambda);
    GpResult out;
    out.iterations = r.iterations;
    out.hpwl = r.hpwl;
    out.overflow = r.overflow;
    out.converged = r.converged != 0;
    out.stagnated = r.stagnated != 0;
    out.rollbackIter = r.rollback_iter;
    out.evaluations = static_cast<long>(r.evaluations);
    const bool noop = out.converged && r.iterations == 0 && stage != GpStage::kFillerOnly;
    if (!noop) {  // an already-converged stage records no rows (eplace.cpp:278-296)
        std::vector<spg_iter_metrics> rows(static_cast<size_t>(std::max(r.iterations, 1)));
        int n = 0;
        check(spg_metrics_d2h(ctx, rows.data(), static_cast<int>(rows.size()), &n));
        s.sink.beginStage(toString(stage));
        for (int i = 0; i < n; ++i) {
            const spg_iter_metrics& d = rows[static_cast<size_t>(i)];
            IterMetrics m;
            m.iter = d.iter;
            m.hpwl = d.hpwl;
            m.overflow = d.overflow;
            m.lambda = d.lambda;
            m.gamma = d.gamma;
            m.step_size = d.step_size;
            m.grad_norm_wl = d.grad_norm_wl;
            m.grad_norm_den = d.grad_norm_den;
            m.max_displacement = d.max_displacement;
            m.elapsed_ms = d.elapsed_ms;
            m.eval_lambda = d.eval_lambda;
            m.eval_gamma = d.eval_gamma;
            m.delta_hpwl = d.delta_hpwl;
            m.lambda_mu = d.lambda_mu;
            m.evaluations = static_cast<long>(d.evaluations);
            s.sink.push(m);
        }
        s.sink.endStage(r.elapsed_ms);
    }
    s.sink.setSummary(prefix + "evaluations", static_cast<double>(out.evaluations));
    s.sink.setSummary(prefix + "converged", out.converged ? 1 : 0);
    s.sink.setSummary(prefix + "stagnated", out.stagnated ? 1 : 0);
    s.sink.setSummary(prefix + "rollback_iter", out.rollbackIter);
    return out;
}

}  // namespace sp
