// C entry points onto the reference's OWN CPU implementation of the GP path, compiled
// from the reference sources (see oracle/Makefile). Test infrastructure only: tests and
// the CPU-baseline leg of the benchmark load it to check and time against; the product
// never links it.
//
// Every function builds or drives reference objects directly:
//   sp::PlaceDB (src/db/place_db.h), sp::BinGrid (src/gp/bin_grid.h),
//   sp::WaWirelength (src/gp/wa_wirelength.h), sp::computeHPWL (src/db/hpwl.h),
//   sp::initializeFillers (src/gp/filler.h), sp::EPlace (src/gp/eplace.h),
//   sp::makeNesterov (src/numeric/optimizer.h), sp::makePoissonBackend
//   (src/numeric/poisson_backend.h; CPU backend = oracle/ref_shim/poisson_shim.cpp).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <exception>
#include <memory>
#include <string>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

#include "db/hpwl.h"
#include "db/place_db.h"
#include "gp/bin_grid.h"
#include "gp/diagnostics.h"
#include "gp/eplace.h"
#include "gp/filler.h"
#include "gp/wa_wirelength.h"
#include "io/bookshelf_reader.h"
#include "io/bookshelf_writer.h"
#include "lg/abacus.h"
#include "lg/macro_sa.h"
#include "numeric/reduction.h"
#include "numeric/optimizer.h"
#include "numeric/poisson_backend.h"
#include "spgpu.h"
#include "util/config.h"
#include "util/invariant.h"
#include "util/logger.h"
#include "util/metrics.h"

namespace {

thread_local std::string g_err;

struct RefDb {
    sp::PlaceDB db;
};

struct RefGrid {
    sp::BinGrid grid;
};

int fail(const std::exception& e) {
    g_err = e.what();
    if (auto* ie = dynamic_cast<const sp::InvariantError*>(&e)) {
        if (ie->kind == "non_finite") return SPG_E_NON_FINITE;
        if (ie->kind == "out_of_core") return SPG_E_OUT_OF_CORE;
        if (ie->kind == "convergence_mismatch") return SPG_E_CONVERGENCE;
        if (ie->kind == "rollback_mismatch") return SPG_E_ROLLBACK;
    }
    return SPG_E_INVALID;
}

void buildDb(sp::PlaceDB& db, const spg_db_view* v) {
    const int total = v->num_nodes + v->num_fillers;
    db.numMovable = v->num_movable;
    db.numNodes = v->num_nodes;
    db.numFillers = v->num_fillers;
    db.reserveNodes(total);
    for (int i = 0; i < total; ++i) {
        db.addNode("o" + std::to_string(i), v->node_w[i], v->node_h[i], v->node_flags[i]);
        db.node_x[static_cast<size_t>(i)] = v->node_x[i];
        db.node_y[static_cast<size_t>(i)] = v->node_y[i];
    }
    db.numPins = v->num_pins;
    db.numNets = v->num_nets;
    db.pin_offset_x.assign(v->pin_offset_x, v->pin_offset_x + v->num_pins);
    db.pin_offset_y.assign(v->pin_offset_y, v->pin_offset_y + v->num_pins);
    db.pin2node.assign(v->pin2node, v->pin2node + v->num_pins);
    db.pin2net.assign(v->pin2net, v->pin2net + v->num_pins);
    db.net2pin_start.assign(v->net2pin_start, v->net2pin_start + v->num_nets + 1);
    db.flat_net2pin.assign(v->flat_net2pin, v->flat_net2pin + v->num_pins);
    db.node2pin_start.assign(v->node2pin_start, v->node2pin_start + total + 1);
    db.flat_node2pin.assign(v->flat_node2pin, v->flat_node2pin + v->num_pins);
    db.net_weight.assign(static_cast<size_t>(v->num_nets), 1.f);
    db.net_name.assign(static_cast<size_t>(v->num_nets), "n");
    for (int r = 0; r < v->num_rows; ++r) {
        sp::PlaceDB::SiteRow row;
        row.ly = v->row_ly[r];
        row.height = v->row_height[r];
        row.lx = v->row_lx[r];
        row.step = v->row_step[r];
        row.numSites = v->row_num_sites[r];
        db.rows.push_back(row);
    }
    db.computeRegions();
}

sp::Config makeConfig(const spg_params* p) {
    sp::Config c;
    c.target_density = p->target_density;
    c.target_overflow = p->target_overflow;
    c.cgp_target_overflow = p->cgp_target_overflow;
    c.gp_max_iter = p->gp_max_iter;
    c.ignore_net_degree = p->ignore_net_degree;
    c.gp_bin_dim = p->gp_bin_dim;
    c.filler_only_iters = p->filler_only_iters;
    c.delta_hpwl_ref = p->delta_hpwl_ref;
    c.lambda_schedule = p->lambda_schedule_relative ? "relative" : "fixed";
    c.delta_hpwl_relative = p->delta_hpwl_relative;
    c.use_bb = p->use_bb != 0;
    c.gp_backtrack = p->gp_backtrack != 0;
    c.gp_stagnation_window = p->gp_stagnation_window;
    c.gp_stagnation_min_gain = p->gp_stagnation_min_gain;
    c.random_seed = p->random_seed;
    c.poisson_backend = "cpu";
    c.verbose = p->verbose != 0;
    return c;
}

}  // namespace

extern "C" {

const char* spref_last_error(void) { return g_err.c_str(); }

void spref_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

int spref_max_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void spref_quiet(int quiet) {
    sp::Logger::get().setLevel(quiet ? sp::LogLevel::kError : sp::LogLevel::kInfo);
}

// ------------------------------------------------------------------ PlaceDB
void* spref_db_create(const spg_db_view* v) {
    try {
        auto* r = new RefDb;
        buildDb(r->db, v);
        return r;
    } catch (const std::exception& e) {
        fail(e);
        return nullptr;
    }
}

void spref_db_destroy(void* h) { delete static_cast<RefDb*>(h); }

// counts[0..4] = numMovable, numNodes, numFillers, numPins, numNets
void spref_db_counts(void* h, int* counts) {
    const sp::PlaceDB& db = static_cast<RefDb*>(h)->db;
    counts[0] = db.numMovable;
    counts[1] = db.numNodes;
    counts[2] = db.numFillers;
    counts[3] = db.numPins;
    counts[4] = db.numNets;
}

// core[0..3] = core lx ly hx hy, core[4] = rowHeight ; area = totalRowArea
void spref_db_regions(void* h, float* core, double* area) {
    const sp::PlaceDB& db = static_cast<RefDb*>(h)->db;
    core[0] = db.coreRegion.lx;
    core[1] = db.coreRegion.ly;
    core[2] = db.coreRegion.hx;
    core[3] = db.coreRegion.hy;
    core[4] = db.rowHeight;
    *area = db.totalRowArea;
}

void spref_db_get_nodes(void* h, float* x, float* y, float* w, float* hh, uint8_t* flags) {
    const sp::PlaceDB& db = static_cast<RefDb*>(h)->db;
    const size_t n = static_cast<size_t>(db.totalNodes());
    if (x) std::memcpy(x, db.node_x.data(), n * sizeof(float));
    if (y) std::memcpy(y, db.node_y.data(), n * sizeof(float));
    if (w) std::memcpy(w, db.node_w.data(), n * sizeof(float));
    if (hh) std::memcpy(hh, db.node_h.data(), n * sizeof(float));
    if (flags) std::memcpy(flags, db.node_flags.data(), n);
}

void spref_db_set_xy(void* h, const float* x, const float* y) {
    sp::PlaceDB& db = static_cast<RefDb*>(h)->db;
    const size_t n = static_cast<size_t>(db.totalNodes());
    std::memcpy(db.node_x.data(), x, n * sizeof(float));
    std::memcpy(db.node_y.data(), y, n * sizeof(float));
}

void spref_db_set_flags(void* h, const uint8_t* flags) {
    sp::PlaceDB& db = static_cast<RefDb*>(h)->db;
    std::memcpy(db.node_flags.data(), flags, static_cast<size_t>(db.totalNodes()));
}

// ------------------------------------------------------------------ fillers
// info[0..5] = count, width, height, whitespaceArea, nodeAreaScaled, totalFillerArea
int spref_fillers_init(void* h, float targetDensity, uint64_t seed, double* info) {
    try {
        sp::PlaceDB& db = static_cast<RefDb*>(h)->db;
        sp::Config cfg;
        cfg.target_density = targetDensity;
        cfg.random_seed = seed;
        const sp::FillerInfo fi = sp::initializeFillers(db, cfg);
        info[0] = fi.count;
        info[1] = fi.width;
        info[2] = fi.height;
        info[3] = fi.whitespaceArea;
        info[4] = fi.nodeAreaScaled;
        info[5] = fi.totalFillerArea;
        return 0;
    } catch (const std::exception& e) {
        return fail(e);
    }
}

int spref_fillers_scatter(void* h, uint64_t seed, uint64_t seedOffset) {
    try {
        sp::PlaceDB& db = static_cast<RefDb*>(h)->db;
        sp::Config cfg;
        cfg.random_seed = seed;
        sp::scatterFillers(db, cfg, seedOffset);
        return 0;
    } catch (const std::exception& e) {
        return fail(e);
    }
}

// ------------------------------------------------------------------ BinGrid
void* spref_grid_create(void* dbh, float targetDensity, int binDim, int chunks) {
    try {
        auto* g = new RefGrid;
        g->grid.initialize(static_cast<RefDb*>(dbh)->db, targetDensity, binDim, chunks, false, 4);
        return g;
    } catch (const std::exception& e) {
        fail(e);
        return nullptr;
    }
}

void spref_grid_destroy(void* g) { delete static_cast<RefGrid*>(g); }

// info[0..4] = dim, stepX, stepY, originX, originY ; den = overflowDenominator
void spref_grid_info(void* g, float* info, double* den) {
    const sp::BinGrid& grid = static_cast<RefGrid*>(g)->grid;
    info[0] = static_cast<float>(grid.dim());
    info[1] = grid.stepX();
    info[2] = grid.stepY();
    info[3] = grid.originX();
    info[4] = grid.originY();
    *den = grid.overflowDenominator();
}

void spref_grid_accumulate(void* g, void* dbh) {
    static_cast<RefGrid*>(g)->grid.accumulate(static_cast<RefDb*>(dbh)->db);
}

float spref_grid_overflow(void* g) { return static_cast<RefGrid*>(g)->grid.overflow(); }

void spref_grid_solve(void* g) { static_cast<RefGrid*>(g)->grid.solveField(); }

void spref_grid_gather(void* g, void* dbh, float* force) {
    static_cast<RefGrid*>(g)->grid.gatherForce(static_cast<RefDb*>(dbh)->db, force);
}

double spref_grid_total_charge(void* g, void* dbh) {
    return static_cast<RefGrid*>(g)->grid.totalCharge(static_cast<RefDb*>(dbh)->db);
}

// which: 0 node, 1 filler, 2 terminal, 3 base, 5 phi, 6 xi_x, 7 xi_y
void spref_grid_read(void* g, int which, float* out) {
    const sp::BinGrid& grid = static_cast<RefGrid*>(g)->grid;
    const std::vector<float>* v = nullptr;
    switch (which) {
        case 0: v = &grid.nodeDensity(); break;
        case 1: v = &grid.fillerDensity(); break;
        case 2: v = &grid.terminalDensity(); break;
        case 3: v = &grid.baseDensity(); break;
        case 5: v = &grid.potential(); break;
        case 6: v = &grid.fieldX(); break;
        case 7: v = &grid.fieldY(); break;
        default: return;
    }
    std::memcpy(out, v->data(), v->size() * sizeof(float));
}

// ------------------------------------------------------------------ WA / HPWL
double spref_wa(void* dbh, float gamma, int ignoreDeg, float* grad) {
    const sp::PlaceDB& db = static_cast<RefDb*>(dbh)->db;
    sp::WaWirelength wa;
    wa.prepare(db);
    double wl = 0.0;
    wa.compute(db, gamma, ignoreDeg, &wl, grad);
    return wl;
}

double spref_hpwl(void* dbh) { return sp::computeHPWL(static_cast<RefDb*>(dbh)->db); }

float spref_gamma(float tau, float binStep) { return sp::computeGamma(tau, binStep); }

// ------------------------------------------------------------------ Poisson
int spref_poisson(int nx, int ny, float sx, float sy, const float* rho, float* phi, float* ex,
                  float* ey) {
    try {
        auto be = sp::makePoissonBackend({nx, ny, sx, sy, false, 4});
        std::vector<float> in(rho, rho + static_cast<size_t>(nx) * ny);
        be->solve({in.data(), nx, ny}, {phi, nx, ny}, {ex, nx, ny}, {ey, nx, ny});
        return 0;
    } catch (const std::exception& e) {
        return fail(e);
    }
}

// Times `rounds` solves after `warm` warm-up solves (tools/poisson_bench/main.cpp:13-33);
// returns milliseconds per solve.
double spref_poisson_bench(int n, int warm, int rounds, int fftwThreads, const float* rho) {
    try {
        auto be = sp::makePoissonBackend({n, n, 1.f, 1.f, false, fftwThreads});
        std::vector<float> in(rho, rho + static_cast<size_t>(n) * n), a(in.size()), b(in.size()),
            c(in.size());
        for (int i = 0; i < warm; ++i) be->solve({in.data(), n, n}, {a.data(), n, n}, {b.data(), n, n}, {c.data(), n, n});
        const double t0 = omp_get_wtime();
        for (int i = 0; i < rounds; ++i) be->solve({in.data(), n, n}, {a.data(), n, n}, {b.data(), n, n}, {c.data(), n, n});
        return (omp_get_wtime() - t0) * 1e3 / rounds;
    } catch (const std::exception& e) {
        fail(e);
        return -1.0;
    }
}

// ------------------------------------------------------------------ EPlace
// One metrics row as the doubles the tests read (sp::IterMetrics, src/util/metrics.h:12-28).
constexpr int kRowWidth = 14;
void putRow(const sp::IterMetrics& row, double* o) {
    o[0] = row.iter;
    o[1] = row.hpwl;
    o[2] = row.overflow;
    o[3] = row.lambda;
    o[4] = row.gamma;
    o[5] = row.step_size;
    o[6] = static_cast<double>(row.evaluations);
    o[7] = row.elapsed_ms;
    o[8] = row.grad_norm_wl;
    o[9] = row.grad_norm_den;
    o[10] = row.eval_lambda;
    o[11] = row.eval_gamma;
    o[12] = row.delta_hpwl;
    o[13] = row.lambda_mu;
}

sp::GpStage toStage(int stage) {
    return stage == SPG_STAGE_MGP ? sp::GpStage::kMGP
         : stage == SPG_STAGE_FILLER_ONLY ? sp::GpStage::kFillerOnly
                                          : sp::GpStage::kCGP;
}

void putResult(const sp::GpResult& r, double ms, double* result) {
    result[0] = r.iterations;
    result[1] = r.hpwl;
    result[2] = r.overflow;
    result[3] = r.converged;
    result[4] = r.stagnated;
    result[5] = r.rollbackIter;
    result[6] = static_cast<double>(r.evaluations);
    result[7] = ms;
}

// result[0..7] = iterations, hpwl, overflow, converged, stagnated, rollbackIter,
//                evaluations, elapsed_ms
// rows: up to cap metrics rows, kRowWidth doubles each (putRow)
int spref_eplace_run(void* dbh, const spg_params* p, int stage, double* result, double* init,
                     double* rows, int cap, int* nRows) {
    try {
        sp::PlaceDB& db = static_cast<RefDb*>(dbh)->db;
        const sp::Config cfg = makeConfig(p);
        sp::MetricsSink sink;
        sp::EPlace engine(db, cfg, sink);
        const sp::GpStage st = toStage(stage);
        sp::GpRunOptions o;
        o.freezeLambda = p->freeze_lambda != 0;
        o.freezeGamma = p->freeze_gamma != 0;
        const double t0 = omp_get_wtime();
        const sp::GpResult r = engine.run(st, o);
        putResult(r, (omp_get_wtime() - t0) * 1e3, result);
        const auto& m = sink.stageMetrics(sp::toString(st));
        int n = 0;
        for (const auto& row : m) {
            if (n >= cap) break;
            putRow(row, rows + kRowWidth * n);
            ++n;
        }
        *nRows = n;
        (void)init;
        return 0;
    } catch (const std::exception& e) {
        return fail(e);
    }
}

// EPlace::run with Config::gp_diagnostics on and the sink writing under `root`: the reference's
// own GP diagnostics of the stage (first_eval, stagnation_mid, last_eval, delivered). result as
// spref_eplace_run's.
int spref_eplace_run_diagnostics(void* dbh, const spg_params* p, int stage, const char* root, double* result) {
    try {
        sp::PlaceDB& db = static_cast<RefDb*>(dbh)->db;
        sp::Config cfg = makeConfig(p);
        cfg.gp_diagnostics = true;
        sp::MetricsSink sink;
        sink.setOutputDir(root);
        sp::EPlace engine(db, cfg, sink);
        const double t0 = omp_get_wtime();
        const sp::GpResult r = engine.run(toStage(stage));
        putResult(r, (omp_get_wtime() - t0) * 1e3, result);
        return 0;
    } catch (const std::exception& e) {
        return fail(e);
    }
}

// diagnoseDelivered (src/gp/diagnostics.cpp:175-191) at the handle's positions: the reference's
// "delivered" GP diagnostic for the stage's opt set (buildOptSet, eplace.cpp:82-94), with the
// opt nodes' previous positions (x then y, opt order; n_prev = 0 for none).
int spref_diagnose_delivered(void* dbh, const spg_params* p, int stage, const char* root, int iter, float lambda,
                             float gamma, int grid_dim, const float* previous, int n_prev) {
    try {
        sp::PlaceDB& db = static_cast<RefDb*>(dbh)->db;
        const sp::Config cfg = makeConfig(p);
        const sp::GpStage st = toStage(stage);
        std::vector<int> opt;
        if (st != sp::GpStage::kFillerOnly)
            for (int i = 0; i < db.numMovable; ++i) {
                if (db.isFixed(i) || db.isNI(i)) continue;
                if (st == sp::GpStage::kCGP && db.isMacro(i)) continue;
                opt.push_back(i);
            }
        for (int i = db.numNodes; i < db.totalNodes(); ++i) opt.push_back(i);
        std::vector<float> prev;
        if (previous && n_prev > 0) prev.assign(previous, previous + n_prev);
        sp::diagnoseDelivered(root, sp::toString(st), iter, lambda, gamma, db, cfg, grid_dim, opt, prev);
        return 0;
    } catch (const std::exception& e) {
        return fail(e);
    }
}

// EPlace::Impl::objAndGrad (src/gp/eplace.cpp:136-203) at opt-set positions pos (x then y, opt
// order of buildOptSet, eplace.cpp:82-94) for the given lambda and gamma, composed from the
// reference's own operators the way objAndGrad composes them: BinGrid built as the EPlace
// constructor builds it (eplace.cpp:207-215), accumulate, overflow, solveField, gatherForce,
// WaWirelength::compute, computeHPWL, then the preconditioned assembly of eplace.cpp:166-189
// and its two fixed-chunk sums. The positions of the opt nodes stay written into the handle.
// out[0..4] = WA value (the objective), tau, HPWL, sum|grad WL|, sum|q xi|. n_out gets nOpt.
int spref_obj_and_grad(void* dbh, const spg_params* p, int stage, float lambda, float gamma, const float* pos,
                       float* grad, double* out, int* n_out) {
    try {
        sp::PlaceDB& db = static_cast<RefDb*>(dbh)->db;
        const sp::Config cfg = makeConfig(p);
        std::vector<int> opt;
        if (stage != SPG_STAGE_FILLER_ONLY) {
            for (int i = 0; i < db.numMovable; ++i) {
                if (db.isFixed(i) || db.isNI(i)) continue;
                if (stage == SPG_STAGE_CGP && db.isMacro(i)) continue;
                opt.push_back(i);
            }
        }
        for (int i = db.numNodes; i < db.totalNodes(); ++i) opt.push_back(i);
        const int n = static_cast<int>(opt.size());
        *n_out = n;
        if (!pos) return 0;
        const int total = db.totalNodes();
        for (int k = 0; k < n; ++k) {
            db.node_x[static_cast<size_t>(opt[static_cast<size_t>(k)])] = pos[k];
            db.node_y[static_cast<size_t>(opt[static_cast<size_t>(k)])] = pos[n + k];
        }
        sp::BinGrid grid;
        grid.initialize(db, cfg.target_density, cfg.gp_bin_dim, cfg.density_chunks, false, cfg.fftw_threads);
        sp::WaWirelength wl;
        wl.prepare(db);
        std::vector<float> force(static_cast<size_t>(2 * total), 0.f);
        std::vector<float> gradWl(static_cast<size_t>(2 * db.numMovable), 0.f);
        grid.accumulate(db);
        const float tau = grid.overflow();
        grid.solveField();
        grid.gatherForce(db, force.data());
        double wlObj = 0.0;
        wl.compute(db, gamma, cfg.ignore_net_degree, &wlObj, gradWl.data());
        const double hpwl = sp::computeHPWL(db);
        const int nMov = db.numMovable;
        const double sumWl = sp::deterministicSumWithWork(n, [&](int64_t kk, double& accWl) {
            const int k = static_cast<int>(kk);
            const int i = opt[static_cast<size_t>(k)];
            const bool hasWl = i < nMov;
            const float wlx = hasWl ? gradWl[static_cast<size_t>(i)] : 0.f;
            const float wly = hasWl ? gradWl[static_cast<size_t>(nMov + i)] : 0.f;
            const float fx = force[static_cast<size_t>(i)];
            const float fy = force[static_cast<size_t>(total + i)];
            const double degree = static_cast<double>(db.nodeDegree(i));
            const float precond =
                static_cast<float>(1.0 / std::max(1.0, degree + static_cast<double>(lambda) * db.area(i)));
            grad[k] = precond * (wlx - lambda * fx);
            grad[n + k] = precond * (wly - lambda * fy);
            if (hasWl) accWl += std::fabs(wlx) + std::fabs(wly);
        });
        const double sumDen = sp::deterministicSum(n, [&](int64_t kk) -> double {
            const int i = opt[static_cast<size_t>(kk)];
            return std::fabs(force[static_cast<size_t>(i)]) + std::fabs(force[static_cast<size_t>(total + i)]);
        });
        out[0] = wlObj;
        out[1] = tau;
        out[2] = hpwl;
        out[3] = sumWl;
        out[4] = sumDen;
        return 0;
    } catch (const std::exception& e) {
        return fail(e);
    }
}

// sp::legalizeMacros (src/lg/macro_sa.cpp:493): the SA macro legalisation GlobalPlaceStage runs
// between mGP and FILLERONLY (src/stages/gp_stage.cpp:128-132); it leaves the macros F_FIXED.
// res[0..5] = numMacros, overlapBefore, overlapAfter, hpwlBefore, hpwlAfter, repaired.
int spref_legalize_macros(void* dbh, const spg_params* p, double* res) {
    try {
        sp::PlaceDB& db = static_cast<RefDb*>(dbh)->db;
        const sp::Config cfg = makeConfig(p);
        sp::MetricsSink sink;
        const sp::MacroSaResult r = sp::legalizeMacros(db, cfg, sink);
        const double v[6] = {double(r.numMacros), r.overlapBefore, r.overlapAfter, r.hpwlBefore, r.hpwlAfter,
                             double(r.repaired)};
        std::memcpy(res, v, sizeof v);
        return 0;
    } catch (const std::exception& e) {
        return fail(e);
    }
}

// The GP stage sequence of GlobalPlaceStage::run for a design with movable macros
// (src/stages/gp_stage.cpp:99-201), on a handle whose fillers are already initialised:
// mGP, legalizeMacros, scatterFillers with seed offset 1, FILLERONLY, cGP, each EPlace built
// anew. res = 3 stage results of 8 (putResult: mGP, FILLERONLY, cGP) then the 6 values of
// spref_legalize_macros.
int spref_gp_four_stage(void* dbh, const spg_params* p, double* res) {
    try {
        sp::PlaceDB& db = static_cast<RefDb*>(dbh)->db;
        const sp::Config cfg = makeConfig(p);
        sp::MetricsSink sink;
        const sp::GpStage order[3] = {sp::GpStage::kMGP, sp::GpStage::kFillerOnly, sp::GpStage::kCGP};
        for (int s = 0; s < 3; ++s) {
            if (s == 1) {
                const sp::MacroSaResult r = sp::legalizeMacros(db, cfg, sink);
                const double v[6] = {double(r.numMacros), r.overlapBefore, r.overlapAfter, r.hpwlBefore,
                                     r.hpwlAfter, double(r.repaired)};
                std::memcpy(res + 24, v, sizeof v);
                sp::scatterFillers(db, cfg, 1);
            }
            const double t0 = omp_get_wtime();
            sp::GpResult r;
            {
                sp::EPlace engine(db, cfg, sink);
                r = engine.run(order[s]);
            }
            putResult(r, (omp_get_wtime() - t0) * 1e3, res + 8 * s);
        }
        return 0;
    } catch (const std::exception& e) {
        return fail(e);
    }
}

// ------------------------------------------------------------------ Nesterov
// Minimises f(x) = 0.5 * sum c_i (x_i - t_i)^2 (test/test_nesterov.cpp:14-27) for `steps`
// steps with the reference optimizer. cfgv = {use_bb, backtrack, init_step}.
// Writes the final positions to pos; out[0..2] = objective, evaluations, step size.
int spref_nesterov_quadratic(int n, const float* coef, const float* target, float* pos,
                             int steps, int useBb, int backtrack, float initStep, double* out) {
    try {
        std::vector<float> c(coef, coef + n), t(target, target + n);
        auto f = [&](const float* x, float* g, double* obj) {
            double o = 0.0;
            for (int i = 0; i < n; ++i) {
                const double d = static_cast<double>(x[i]) - t[static_cast<size_t>(i)];
                o += 0.5 * c[static_cast<size_t>(i)] * d * d;
                g[i] = static_cast<float>(c[static_cast<size_t>(i)] * d);
            }
            *obj = o;
        };
        sp::OptConfig cfg;
        cfg.use_bb = useBb != 0;
        cfg.backtrack = backtrack != 0;
        cfg.init_step = initStep;
        auto opt = sp::makeNesterov(f, nullptr, cfg);
        for (int k = 0; k < steps; ++k) opt->step(pos, n);
        out[0] = opt->objective();
        out[1] = static_cast<double>(opt->evaluations());
        out[2] = opt->stepSize();
        return 0;
    } catch (const std::exception& e) {
        return fail(e);
    }
}

// ------------------------------------------------------------------ BookShelf
// sp::BookshelfReader::read (src/io/bookshelf_reader.cpp) into a new PlaceDB handle.
void* spref_bookshelf_read(const char* aux) {
    try {
        auto* r = new RefDb;
        sp::BookshelfReader reader;
        reader.read(aux, r->db);
        return r;
    } catch (const std::exception& e) {
        fail(e);
        return nullptr;
    }
}

// counts[0..3] = rows, bytes of node names, bytes of net names (NUL-terminated, back to back)
void spref_db_more_counts(void* h, long long* counts) {
    const sp::PlaceDB& db = static_cast<RefDb*>(h)->db;
    long long a = 0, b = 0;
    for (const std::string& s : db.node_name) a += static_cast<long long>(s.size()) + 1;
    for (const std::string& s : db.net_name) b += static_cast<long long>(s.size()) + 1;
    counts[0] = static_cast<long long>(db.rows.size());
    counts[1] = a;
    counts[2] = b;
}

void spref_db_get_pins(void* h, float* ox, float* oy, int* pin2node, int* pin2net, int* net2pin_start,
                       int* flat_net2pin, int* node2pin_start, int* flat_node2pin) {
    const sp::PlaceDB& db = static_cast<RefDb*>(h)->db;
    const size_t p = db.pin2node.size();
    std::memcpy(ox, db.pin_offset_x.data(), p * sizeof(float));
    std::memcpy(oy, db.pin_offset_y.data(), p * sizeof(float));
    std::memcpy(pin2node, db.pin2node.data(), p * sizeof(int));
    std::memcpy(pin2net, db.pin2net.data(), p * sizeof(int));
    std::memcpy(net2pin_start, db.net2pin_start.data(), db.net2pin_start.size() * sizeof(int));
    std::memcpy(flat_net2pin, db.flat_net2pin.data(), p * sizeof(int));
    std::memcpy(node2pin_start, db.node2pin_start.data(), db.node2pin_start.size() * sizeof(int));
    std::memcpy(flat_node2pin, db.flat_node2pin.data(), p * sizeof(int));
}

void spref_db_get_rows(void* h, float* ly, float* height, float* lx, float* step, int* sites) {
    const sp::PlaceDB& db = static_cast<RefDb*>(h)->db;
    for (size_t r = 0; r < db.rows.size(); ++r) {
        ly[r] = db.rows[r].ly;
        height[r] = db.rows[r].height;
        lx[r] = db.rows[r].lx;
        step[r] = db.rows[r].step;
        sites[r] = db.rows[r].numSites;
    }
}

void spref_db_get_names(void* h, char* node_names, char* net_names, unsigned char* orient, float* weight) {
    const sp::PlaceDB& db = static_cast<RefDb*>(h)->db;
    for (const std::string& s : db.node_name) {
        std::memcpy(node_names, s.c_str(), s.size() + 1);
        node_names += s.size() + 1;
    }
    for (const std::string& s : db.net_name) {
        std::memcpy(net_names, s.c_str(), s.size() + 1);
        net_names += s.size() + 1;
    }
    std::memcpy(orient, db.node_orient.data(), db.node_orient.size());
    std::memcpy(weight, db.net_weight.data(), db.net_weight.size() * sizeof(float));
}

// sp::legalizeCells (src/lg/abacus.cpp) on the handle's PlaceDB. res[0..9] = preconditionOk,
// cells, failed, rows, segments, roundedWidths, selfcheckOverlaps, selfcheckOffSite, dispMean,
// dispMax.
int spref_abacus(void* h, int area_weight, int reference_trials, double* res) {
    try {
        sp::AbacusOptions o;
        o.areaWeight = area_weight != 0;
        o.referenceTrials = reference_trials != 0;
        const sp::AbacusResult r = sp::legalizeCells(static_cast<RefDb*>(h)->db, o);
        const double v[10] = {double(r.preconditionOk), double(r.cells), double(r.failed), double(r.rows),
                              double(r.segments), double(r.roundedWidths), double(r.selfcheckOverlaps),
                              double(r.selfcheckOffSite), r.dispMean, r.dispMax};
        std::memcpy(res, v, sizeof v);
        return 0;
    } catch (const std::exception& e) {
        return fail(e);
    }
}

// sp::BookshelfReader::readPlacement (src/io/bookshelf_reader.cpp) into the handle's PlaceDB.
int spref_read_placement(void* h, const char* path) {
    try {
        sp::BookshelfReader reader;
        reader.readPlacement(path, static_cast<RefDb*>(h)->db);
        return 0;
    } catch (const std::exception& e) {
        return fail(e);
    }
}

// sp::BookshelfWriter::writePl (src/io/bookshelf_writer.cpp) of the handle's PlaceDB.
int spref_write_pl(void* h, const char* path) {
    try {
        sp::BookshelfWriter::writePl(path, static_cast<RefDb*>(h)->db);
        return 0;
    } catch (const std::exception& e) {
        return fail(e);
    }
}

}  // extern "C"
