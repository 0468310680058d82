// Host side of the implicit energy-conserving orbit-averaged GM-HC-CN method
// (UPIC_METHOD_CN_ORBIT): state, start-up, the outer Anderson/Picard
// iteration on the mesh current, and diagnostics.
//
// Reference: Project3/ec_pic_nyquist_projected.cpp.  The outer iteration
// restates nonlinear_step_uniform_subcycled (:5878) for the level-one
// particle layout that nonlinear_step_orbit (:6477) uses: map evaluations
// J -> J_map run on the GPU (api: eval_map), the small dense Anderson solve
// and the acceptance logic run here, with every vector reduction computed on
// the device in double-double in a fixed order.
//
// HBM layout (N nodes, np particles): particle SoA x2 {x, y, P(3), v(3),
// v_prev(3), vbar(3), id[, q, m]}; state spectra phi, psi, rho, A(3), U(3)
// and their trial copies (2 x 9 complex per node); map records (8 doubles per
// node: grad phi_mid, A^n, A^{n+1}); node currents J, J_field, guesses,
// map values and the Anderson history (3 doubles per node each).
#include <algorithm>
#include <cfloat>
#include <cstdio>
#include <climits>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "context.h"
#include "guess_net.h"
#include "implicit_kernels.h"
#include "upic_common.cuh"

using namespace upic;

namespace upic_host {

constexpr int kHist = 5;         // Anderson memory + 1 (memory <= 4)
constexpr int kNormGrid = 296;
constexpr int kMaxImplicitChunk = 1024;

struct ImplicitState {
    int order = 2, nq = 8, mnq = 8;
    double* qtab = nullptr;  // Gauss rules (ImplicitMapArgs::qtab)
    double dx = 0, dy = 0, dV = 0;
    // particles: two sorted copies (the second is the sort / trial target)
    ParticleSoA P[2];
    double *bx[2] = {}, *by[2] = {}, *bz[2] = {};
    int cur = 0;
    long np = 0, cap = 0;
    bool uniform = true;
    double q0 = 0, m0 = 0, qabs = 0;
    // fields
    double2* spec = nullptr;      // state spectra (9 x N)
    double2* spec_out = nullptr;  // trial spectra (9 x N)
    double2* Jhat = nullptr;      // 3 x N
    double2* gspec = nullptr;     // 5 x N
    double2* dspec = nullptr;     // 10 x N
    double* dreal = nullptr;      // 10 x N
    double* rec = nullptr;        // 8 x N
    unsigned char* excl = nullptr;
    unsigned long long* acc = nullptr;  // 8 x N (J 3 comps + rho)
    double* J = nullptr;          // state current (3 x N)
    double* Jf = nullptr;         // projected current guess (3 x N)
    double* guess = nullptr;
    double* map = nullptr;
    double* trial = nullptr;
    double* trial_map = nullptr;
    double* cand = nullptr;
    double* resid = nullptr;
    double* hx[kHist] = {};
    double* hr[kHist] = {};
    int hcount = 0;
    double* partials = nullptr;
    NormSums* dnorm = nullptr;
    NormSums* hnorm = nullptr;    // pinned
    MapStats* dstats = nullptr;
    MapStats* hstats = nullptr;   // pinned
    int* dflag = nullptr;
    int* hflag = nullptr;         // pinned
    double* ddots = nullptr;
    double* hdots = nullptr;      // pinned (32)
    double scaleJ[4] = {1, 1, 1, 1};
    TileGeom tg{};
    SortWork sw{};
    int grid = 148;
    long steps = 0;
    // kernel-level orbit entry points: host-array staging (grown on demand)
    long ocap = 0;
    double *ox = nullptr, *oy = nullptr, *odx = nullptr, *ovb = nullptr, *oq = nullptr, *ogat = nullptr,
           *ograd = nullptr;
    double* ogrid = nullptr;  // mesh, A^n, A^{n+1}: 9 x N
    int* oerr = nullptr;
    // step diagnostics (grown on first use)
    double2* sd_spec = nullptr;             // 12 x N
    double* sd_rec = nullptr;               // 12 doubles per node
    unsigned long long* sd_counts = nullptr;  // 4
    // field and kinetic energy of the current state, when known
    bool energy_valid = false;
    double energy_W = 0.0, energy_K = 0.0;
    // non-relativistic Picard method (UPIC_METHOD_CN_ORBIT_NONREL)
    bool picard = false;
    double *gx = nullptr, *gy = nullptr, *gz = nullptr;  // velocity guess (sorted order)
    // orbit velocities handed from the solve launch to the deposit launch of
    // a map evaluation (ImplicitMapArgs::vbar_*; relativistic method only)
    double *hvx = nullptr, *hvy = nullptr, *hvz = nullptr;
    // initial A and U (6 x N) for the next start-up (upic_set_initial_potential)
    double* init_AU = nullptr;
    bool init_AU_set = false;
    double* Jprev = nullptr;                              // 3 x N
    // current of the step before the last (UPIC_PREDICTOR_EXTRAPOLATED)
    double* Jold = nullptr;                               // 3 x N
    bool have_Jold = false;
    // local_warm_start: gx/gy/gz keep the orbit velocities of the last map
    // evaluation of the current step
    bool warm_valid = false;
    // selective particle sub-cycling (selective_particle_fallback): substeps
    // per sorted particle (device and host), the refined list, the failing
    // particles of the last map evaluation
    int *nsub = nullptr, *refined = nullptr, *failed = nullptr, *nfailed = nullptr;
    std::vector<int> h_nsub;
    bool layout_active = false;
    int nref = 0, last_refined = 0;
    // sub-orbit records (x0, y0, vbar) of the refined particles, written by
    // the final map evaluation of a sub-cycled step and read by its step
    // diagnostics; roff[i] is refined particle i's first record
    int* roff = nullptr;
    double* sub_rec = nullptr;
    long sub_cap = 0;
    long total_substeps = 0;
    // first guess of the outer current iteration: J0 the guess of the
    // current step; Jx = 2 J^n - J^(n-1) (extrapolated and learned
    // predictors); Jl the learned prediction and the network with its field
    // frames (learned predictor; fbuf: A and phi of the accepted state)
    double *J0 = nullptr, *Jx = nullptr, *Jl = nullptr, *fbuf = nullptr;
    bool have_Jx = false, have_Jl = false, use_learned = false;
    int predictor_used = UPIC_PREDICTOR_PREVIOUS;
    long trained_steps = 0;
    upic::gnet::Net* net = nullptr;
    double* dloss = nullptr;
    NormSums* dnorm3 = nullptr;
    NormSums* hnorm3 = nullptr;  // pinned (3)
    double* hloss = nullptr;     // pinned
    unsigned long long* pstat = nullptr;                  // path statistics counters (4)
    int* perr = nullptr;
    double vb_limit = 0.0;  // bound on |vbar| components of the fixed-point deposit
    double dt_max = 0.0;    // dt at creation: the deposit window guard covers kappa * dt_max
    bool loaded = false;  // upic_set_particles has succeeded
    bool ready = false;   // upic_init_fields has succeeded
    // secant contraction sums of each outer iteration: |x_k - x_{k-1}|^2 at
    // 4 k, |G(x_k) - G(x_{k-1})|^2 at 4 k + 2 (device; pinned copy)
    double* dcon = nullptr;
    double* hcon = nullptr;
    // map evaluations of the current upic_step_implicit call
    // (UPIC_MAPLOG_COUNT values each, upic_map_log)
    std::vector<double> maplog;
    int log_step = 0, map_eval = 0;
    // failed-particle records of the selective layout's failing map
    // evaluations in the current upic_step_implicit call (UPIC_FAILLOG_COUNT
    // values each, upic_failed_particle_log); fail_event: first row of the
    // last event; layout_restart: the step's current layout refinement
    std::vector<double> faillog;
    size_t fail_event = 0;
    int layout_restart = 0;
    double* dfail = nullptr;  // kFailRec doubles per failed particle (grown on demand)
    int dfail_cap = 0;
    // F18: phi, psi, rho, A, U, J, E, B on the grid for upic_probe_fields;
    // probe staging (grown on demand)
    double* probe_grid = nullptr;
    double *px = nullptr, *py = nullptr, *pout = nullptr;
    long pcap = 0;
};

namespace {

// Gauss-Legendre nodes and weights on [0,1] by Newton iteration on the
// Legendre polynomial from the Chebyshev-like start cos(pi (i+3/4)/(n+1/2)),
// the scheme of gauss_legendre_01 (ec_pic_nyquist_projected.cpp:2479).
void gauss_legendre_01(int n, std::vector<double>& s, std::vector<double>& w) {
    s.assign(n, 0.0);
    w.assign(n, 0.0);
    auto legendre = [&](double x, double& pn, double& dp) {
        double p0 = 1.0, p1 = x;
        if (n == 0) { pn = 1.0; dp = 0.0; return; }
        if (n == 1) { pn = x; dp = 1.0; return; }
        for (int k = 2; k <= n; ++k) {
            const double pk = ((2.0 * k - 1.0) * x * p1 - (k - 1.0) * p0) / (double)k;
            p0 = p1;
            p1 = pk;
        }
        pn = p1;
        dp = (double)n * (x * p1 - p0) / (x * x - 1.0);
    };
    const int m = (n + 1) / 2;
    for (int i = 0; i < m; ++i) {
        double x = std::cos(kPi * ((double)i + 0.75) / ((double)n + 0.5));
        for (int it = 0; it < 80; ++it) {
            double pn, dp;
            legendre(x, pn, dp);
            const double d = -pn / dp;
            x += d;
            if (std::fabs(d) < 1.0e-15) break;
        }
        double pn, dp;
        legendre(x, pn, dp);
        const double wt = 2.0 / ((1.0 - x * x) * dp * dp);
        s[i] = 0.5 * (1.0 - x);
        w[i] = 0.5 * wt;
        s[n - 1 - i] = 0.5 * (1.0 + x);
        w[n - 1 - i] = 0.5 * wt;
    }
}

// solve_small_dense_system (ec_pic_nyquist_projected.cpp:5706): Gaussian
// elimination with partial pivoting and the reference's singularity tests.
bool solve_small_dense(std::vector<std::vector<double>> A, std::vector<double> b, std::vector<double>& x) {
    const int n = (int)b.size();
    double scale = 0.0;
    for (const auto& row : A)
        for (double v : row) scale = std::max(scale, std::fabs(v));
    if (!(scale > 0.0) || !std::isfinite(scale)) return false;
    double largest = 0.0, smallest = INFINITY;
    for (int col = 0; col < n; ++col) {
        int pr = col;
        for (int r = col + 1; r < n; ++r)
            if (std::fabs(A[r][col]) > std::fabs(A[pr][col])) pr = r;
        const double piv = std::fabs(A[pr][col]);
        if (!std::isfinite(piv) || piv <= 100.0 * DBL_EPSILON * scale) return false;
        largest = std::max(largest, piv);
        smallest = std::min(smallest, piv);
        if (pr != col) {
            std::swap(A[pr], A[col]);
            std::swap(b[pr], b[col]);
        }
        for (int r = col + 1; r < n; ++r) {
            const double f = A[r][col] / A[col][col];
            for (int j = col; j < n; ++j) A[r][j] -= f * A[col][j];
            b[r] -= f * b[col];
        }
    }
    if (smallest <= 1.0e-12 * largest) return false;
    x.assign(n, 0.0);
    for (int r = n - 1; r >= 0; --r) {
        double rhs = b[r];
        for (int j = r + 1; j < n; ++j) rhs -= A[r][j] * x[j];
        x[r] = rhs / A[r][r];
        if (!std::isfinite(x[r])) return false;
    }
    return true;
}

struct Norms {
    double rms_relative = INFINITY, max_relative = INFINITY, rms_absolute = INFINITY;
    double rms_scaled = INFINITY, max_scaled = INFINITY;
};

bool is_even_nyquist(int i, int n) { return n > 1 && n % 2 == 0 && i == n / 2; }

int alloc_particles(upic_ctx* c, ImplicitState& s, long cap, bool with_qm) {
    int rc;
    for (int k = 0; k < 2; ++k) {
        if ((rc = alloc_soa(c, s.P[k], cap, true, with_qm))) return rc;
        if ((rc = dalloc(c, &s.bx[k], cap)) || (rc = dalloc(c, &s.by[k], cap)) || (rc = dalloc(c, &s.bz[k], cap)))
            return rc;
    }
    if ((s.picard || c->cfg.local_warm_start) &&
        ((rc = dalloc(c, &s.gx, cap)) || (rc = dalloc(c, &s.gy, cap)) || (rc = dalloc(c, &s.gz, cap))))
        return rc;
    if (!s.picard &&
        ((rc = dalloc(c, &s.hvx, cap)) || (rc = dalloc(c, &s.hvy, cap)) || (rc = dalloc(c, &s.hvz, cap))))
        return rc;
    if (c->cfg.selective_particle_fallback &&
        ((rc = dalloc(c, &s.nsub, cap)) || (rc = dalloc(c, &s.refined, cap)) || (rc = dalloc(c, &s.roff, cap))))
        return rc;
    // the failing particles of a map evaluation, for the failed-particle log
    if (!s.picard && ((rc = dalloc(c, &s.failed, cap)) || (rc = dalloc(c, &s.nfailed, 1)))) return rc;
    if ((rc = alloc_sortwork(c, s.sw, cap, s.tg))) return rc;
    s.cap = cap;
    return ensure_tmp3(c, cap);
}

void free_particles(upic_ctx* c, ImplicitState& s) {
    for (int k = 0; k < 2; ++k) {
        free_soa(c, s.P[k]);
        dfree(c, s.bx[k]);
        dfree(c, s.by[k]);
        dfree(c, s.bz[k]);
        s.bx[k] = s.by[k] = s.bz[k] = nullptr;
    }
    dfree(c, s.gx);
    dfree(c, s.gy);
    dfree(c, s.gz);
    s.gx = s.gy = s.gz = nullptr;
    dfree(c, s.hvx);
    dfree(c, s.hvy);
    dfree(c, s.hvz);
    s.hvx = s.hvy = s.hvz = nullptr;
    dfree(c, s.nsub);
    dfree(c, s.refined);
    dfree(c, s.failed);
    dfree(c, s.nfailed);
    dfree(c, s.roff);
    dfree(c, s.sub_rec);
    s.nsub = s.refined = s.failed = s.nfailed = s.roff = nullptr;
    s.sub_rec = nullptr;
    s.sub_cap = 0;
    free_sortwork(c, s.sw);
    s.cap = 0;
}

// Sort the active set by cell of x (shift 0) and make the sorted copy active.
int sort_active(upic_ctx* c, ImplicitState& s) {
    ParticleSoA& src = s.P[s.cur];
    ParticleSoA& dst = s.P[1 - s.cur];
    UPIC_CUDA(c, sort_particles_by_tile(s.tg, src, s.np, c->cfg.Lx, c->cfg.Ly, 0.0, s.sw, c->st));
    UPIC_CUDA(c, permute_particles(src, dst, s.np, s.sw, c->st));
    // vbar arrays ride along through the spare velocity slots of a temporary SoA
    ParticleSoA vs{}, vd{};
    vs.vx = s.bx[s.cur];
    vs.vy = s.by[s.cur];
    vs.vz = s.bz[s.cur];
    vd.vx = s.bx[1 - s.cur];
    vd.vy = s.by[1 - s.cur];
    vd.vz = s.bz[1 - s.cur];
    UPIC_CUDA(c, permute_particles(vs, vd, s.np, s.sw, c->st));
    s.cur = 1 - s.cur;
    return 0;
}

// One evaluation of the outer map at `guess` (evaluate_selective_current_map_at_layout
// :5235 with every particle at level one).  Result in `out` (3 x N).  With
// write_state the particles' trial end state goes to the spare set and the
// trial spectra to spec_out.  Returns UPIC_ERR_LOCAL_PARTICLE when a local
// solve fails (the step then fails, as SelectiveParticleRefinementNeeded
// propagates in the reference), with the failure described in c->err.
int launch_residual_sums(upic_ctx* c, ImplicitState& s, const double* map, const double* guess);
void norms_from_sums(upic_ctx* c, ImplicitState& s, Norms& n);

// One evaluation of the outer map at `guess` into `out`.  With norms set, the
// residual norms of (out, guess) are formed in the same round trip to the
// host as the map's statistics.
// One row of upic_map_log for a map evaluation with statistics m
// (nonlinear_step_uniform_subcycled's particle-history record :5918-5945).
void log_map_evaluation(ImplicitState& s, const MapStats& m) {
    double worst;
    std::memcpy(&worst, &m.worst_scaled_bits, sizeof(double));
    if (!std::isfinite(worst) || worst >= 1.0e300) worst = INFINITY;  // the kernels record non-finite as 1e300
    const bool ok = m.failures == 0;
    const double mean = s.total_substeps > 0 ? (double)m.iter_total / (double)s.total_substeps : 0.0;
    const double row[UPIC_MAPLOG_COUNT] = {(double)s.log_step, (double)++s.map_eval, ok ? 1.0 : 0.0,
                                           (double)m.failures, worst, ok ? mean : NAN, (double)m.iter_max};
    s.maplog.insert(s.maplog.end(), row, row + UPIC_MAPLOG_COUNT);
}

// Records of the failed particles of the map evaluation just run with
// arguments a (the selective layout's): each failing local solve is run
// again on the evaluation's fields with its report (failure_report_kernel),
// the rows sorted by particle index as the reference sorts its list
// (:5402-5406) and appended to the call's failed-particle log.
int record_failures(upic_ctx* c, ImplicitState& s, const ImplicitMapArgs& a) {
    int nf = 0;
    UPIC_CUDA(c, cudaMemcpyAsync(&nf, s.nfailed, sizeof(int), cudaMemcpyDeviceToHost, c->st));
    int rc = sync(c);
    if (rc) return rc;
    s.fail_event = s.faillog.size();
    if (nf <= 0) return 0;
    if (nf > s.dfail_cap) {
        dfree(c, s.dfail);
        s.dfail = nullptr;
        s.dfail_cap = 0;
        if ((rc = dalloc(c, &s.dfail, (size_t)kFailRec * nf))) return rc;
        s.dfail_cap = nf;
    }
    UPIC_CUDA(c, launch_failure_report(s.order, s.uniform, a.split != 0, s.tg, a, s.failed, nf, s.dfail, c->st));
    std::vector<double> rows((size_t)kFailRec * nf);
    UPIC_CUDA(c, cudaMemcpyAsync(rows.data(), s.dfail, sizeof(double) * rows.size(), cudaMemcpyDeviceToHost, c->st));
    if ((rc = sync(c))) return rc;
    std::vector<int> order(nf);
    for (int i = 0; i < nf; ++i) order[i] = i;
    std::sort(order.begin(), order.end(), [&](int i, int j) { return rows[(size_t)i * kFailRec] < rows[(size_t)j * kFailRec]; });
    for (int i : order) {
        const double head[5] = {(double)s.log_step, (double)s.layout_restart, (double)s.map_eval, 0.0, (double)nf};
        s.faillog.insert(s.faillog.end(), head, head + 5);
        const double* r = rows.data() + (size_t)i * kFailRec;
        s.faillog.insert(s.faillog.end(), r, r + kFailRec);
    }
    return 0;
}

int eval_map(upic_ctx* c, ImplicitState& s, const double* guess, double* out, bool write_state,
             MapStats* stats_out, bool* map_finite = nullptr, Norms* norms = nullptr) {
    const upic_config& cf = c->cfg;
    const int N = c->N;
    // J_field = projected guess (:5264-5265), its spectra
    UPIC_CUDA(c, cudaMemcpyAsync(s.Jf, guess, sizeof(double) * 3 * N, cudaMemcpyDeviceToDevice, c->st));
    if (cf.nyquist_projection) UPIC_CUDA(c, launch_project_nyquist(s.Jf, 3, c->nx, c->ny, c->st));
    UPIC_CUDA(c, fft2d_batched(c->plan, s.Jhat, 3, 0, c->st, s.Jf));
    // continuity + CN update + grad phi_mid and A^{n+1} spectra
    CnArgs k{};
    k.nx = c->nx;
    k.ny = c->ny;
    k.N = N;
    k.kx = c->d_kx;
    k.ky = c->d_ky;
    k.k2 = c->d_k2;
    k.excl = cf.nyquist_projection ? s.excl : nullptr;
    k.Jhat = s.Jhat;
    k.st = s.spec;
    k.out = s.spec_out;
    k.gspec = s.gspec;
    k.dt = cf.dt;
    k.kappa = cf.kappa;
    k.sigma1 = cf.sigma1;
    k.sigma2 = cf.sigma2;
    UPIC_CUDA(c, launch_cn_kspace(k, c->st));
    UPIC_CUDA(c, fft2d_batched(c->plan, s.gspec, 2, 1, c->st, nullptr, 2, s.rec, kIRec, kIRecGpm));
    UPIC_CUDA(c, fft2d_batched(c->plan, s.gspec + 2 * (size_t)N, 3, 1, c->st, nullptr, 2, s.rec, kIRec, kIRecAe));
    // particles: local fixed points and the orbit-averaged deposit
    UPIC_CUDA(c, cudaMemsetAsync(s.acc, 0, sizeof(unsigned long long) * 6 * (size_t)N, c->st));
    UPIC_CUDA(c, cudaMemsetAsync(s.dstats, 0, sizeof(MapStats), c->st));
    UPIC_CUDA(c, cudaMemsetAsync(&s.dstats->first_fail_key, 0xff, sizeof(unsigned long long), c->st));
    const ParticleSoA& p = s.P[s.cur];
    const ParticleSoA& o = s.P[1 - s.cur];
    ImplicitMapArgs a{};
    a.x = p.x; a.y = p.y; a.Px = p.Px; a.Py = p.Py; a.Pz = p.Pz; a.vx = p.vx; a.vy = p.vy; a.vz = p.vz;
    a.q = p.q; a.m = p.m; a.q0 = s.q0; a.m0 = s.m0; a.id = p.id;
    a.ox = o.x; a.oy = o.y; a.oPx = o.Px; a.oPy = o.Py; a.oPz = o.Pz; a.ovx = o.vx; a.ovy = o.vy; a.ovz = o.vz;
    a.obx = s.bx[1 - s.cur]; a.oby = s.by[1 - s.cur]; a.obz = s.bz[1 - s.cur];
    a.np = s.np;
    a.write_state = write_state ? 1 : 0;
    a.Lx = cf.Lx; a.Ly = cf.Ly; a.inv_dx = 1.0 / s.dx; a.inv_dy = 1.0 / s.dy; a.inv_dV = 1.0 / s.dV;
    a.dt = cf.dt; a.kappa = cf.kappa;
    a.rec = s.rec;
    a.split = cf.split_orbit_at_knots;
    a.loc_rtol = cf.local_rtol; a.loc_atol = cf.local_atol; a.loc_damp = cf.local_damping;
    a.loc_maxit = cf.local_max_iter;
    a.chunks = s.sw.chunks;
    a.nchunks = s.sw.nchunks;
    a.acc = s.acc;
    for (int d = 0; d < 3; ++d) a.scale[d] = s.scaleJ[d];
    a.stats = s.dstats;
    a.qtab = s.qtab;
    a.nq = s.nq;
    a.mnq = s.mnq;
    if (s.layout_active) {
        a.nsub = s.nsub;
        a.refined = s.refined;
        a.nref = s.nref;
        a.grid_nx = c->nx;
        a.grid_ny = c->ny;
        a.roff = s.roff;
        a.sub_rec = s.sub_rec;
    }
    if (s.failed) {
        a.failed = s.failed;
        a.nfailed = s.nfailed;
        UPIC_CUDA(c, cudaMemsetAsync(s.nfailed, 0, sizeof(int), c->st));
    }
    a.vbar_x = s.hvx;
    a.vbar_y = s.hvy;
    a.vbar_z = s.hvz;
    if (cf.local_warm_start) {
        if (s.warm_valid) {
            a.warm_x = s.gx;
            a.warm_y = s.gy;
            a.warm_z = s.gz;
        }
        a.keep_x = s.gx;
        a.keep_y = s.gy;
        a.keep_z = s.gz;
    }
    if (s.np > 0) {
        cudaEvent_t e0 = nullptr, e1 = nullptr;
        if (c->profiling) {
            UPIC_CUDA(c, cudaEventCreate(&e0));
            UPIC_CUDA(c, cudaEventCreate(&e1));
            UPIC_CUDA(c, cudaEventRecord(e0, c->st));
        }
        UPIC_CUDA(c, launch_implicit_map(s.order, s.uniform, a.split != 0, s.tg, a, s.grid, c->st));
        if (c->profiling) {
            UPIC_CUDA(c, cudaEventRecord(e1, c->st));
            c->prof_events.emplace_back(e0, e1);
        }
        if (s.layout_active && s.nref > 0) UPIC_CUDA(c, launch_refined_map(s.order, s.uniform, a, c->st));
    }
    UPIC_CUDA(c, launch_convert_acc(s.acc, N, s.scaleJ, out, nullptr, 0.0, 1, c->st));
    if (cf.nyquist_projection) UPIC_CUDA(c, launch_project_nyquist(out, 3, c->nx, c->ny, c->st));
    UPIC_CUDA(c, cudaMemcpyAsync(s.hstats, s.dstats, sizeof(MapStats), cudaMemcpyDeviceToHost, c->st));
    if (map_finite) {
        UPIC_CUDA(c, cudaMemsetAsync(s.dflag, 0, sizeof(int), c->st));
        UPIC_CUDA(c, launch_nonfinite_flag(3 * N, out, s.dflag, c->st));
        UPIC_CUDA(c, cudaMemcpyAsync(s.hflag, s.dflag, sizeof(int), cudaMemcpyDeviceToHost, c->st));
    }
    if (norms) {
        const int rn = launch_residual_sums(c, s, out, guess);
        if (rn) return rn;
    }
    int rc = sync(c);
    if (rc) return rc;
    if (stats_out) *stats_out = *s.hstats;
    if (map_finite) *map_finite = *s.hflag == 0;
    if (norms) norms_from_sums(c, s, *norms);
    log_map_evaluation(s, *s.hstats);
    if (s.hstats->failures > 0) {
        // the selective layout's failures, or the failures that end the step
        // when there is no fallback (the reference's full-step layout)
        if ((s.layout_active || !cf.selective_particle_fallback) && (rc = record_failures(c, s, a))) return rc;
        static const char* names[] = {"none", "nonfinite_map", "superluminal_map", "nonfinite_iterate",
                                      "superluminal_iterate", "maximum_iterations", "too_many_knot_crossings"};
        const unsigned long long key = s.hstats->first_fail_key;
        const int reason = (int)(key & 0xffu);
        char buf[256];
        std::snprintf(buf, sizeof(buf),
                      "local particle solve failed for %d particles (first: particle %llu, %s; "
                      "local_max_iter=%d)",
                      s.hstats->failures, key >> 8, reason < 7 ? names[reason] : "?", cf.local_max_iter);
        return fail(c, UPIC_ERR_LOCAL_PARTICLE, buf);
    }
    if (cf.local_warm_start) s.warm_valid = true;
    return 0;
}

int path_stats(upic_ctx* c, ImplicitState& s, double* out3);

// relative_rms_error_vec_particles / relative_rms_error_vecfield
// (ec_pic_serial_demo.cpp:188, :196) from double-double sums over `count`
// components: r2 = |a - b|^2, map2 = |a|^2, guess2 = |b|^2.
double relative_rms(const NormSums& h, double count) {
    const double cnt = std::max(1.0, count);
    const double rd = std::sqrt((h.r2[0] + h.r2[1]) / cnt);
    const double ra = std::sqrt((h.map2[0] + h.map2[1]) / cnt);
    const double rb = std::sqrt((h.guess2[0] + h.guess2[1]) / cnt);
    return rd / (0.5 * (ra + rb) + 1.0e-300);
}

// One evaluation of the Picard map at the velocity guess (s.gx, s.gy, s.gz):
// evaluate_picard_map_orbit (ec_pic_serial_demo.cpp:1455).  Jbar lands in
// s.map, the trial state in the spare particle set and spec_out; vel: the
// velocity-change sums.
int picard_eval(upic_ctx* c, ImplicitState& s, NormSums& vel) {
    const upic_config& cf = c->cfg;
    const int N = c->N;
    const ParticleSoA& p = s.P[s.cur];
    const ParticleSoA& o = s.P[1 - s.cur];
    // Jbar: orbit-averaged deposit of vbar = (v_guess + v^n) / 2 (:1468-1472)
    UPIC_CUDA(c, cudaMemsetAsync(s.acc, 0, sizeof(unsigned long long) * 6 * (size_t)N, c->st));
    UPIC_CUDA(c, cudaMemsetAsync(s.dstats, 0, sizeof(MapStats), c->st));
    UPIC_CUDA(c, cudaMemsetAsync(&s.dstats->first_fail_key, 0xff, sizeof(unsigned long long), c->st));
    UPIC_CUDA(c, cudaMemsetAsync(s.perr, 0, sizeof(int), c->st));
    if (s.np > 0) {
        ImplicitMapArgs a{};
        a.x = p.x; a.y = p.y; a.vx = p.vx; a.vy = p.vy; a.vz = p.vz;
        a.q = p.q; a.q0 = s.q0; a.id = p.id;
        a.gx = s.gx; a.gy = s.gy; a.gz = s.gz;
        a.vb_limit = s.vb_limit;
        a.np = s.np;
        a.Lx = cf.Lx; a.Ly = cf.Ly; a.inv_dx = 1.0 / s.dx; a.inv_dy = 1.0 / s.dy; a.inv_dV = 1.0 / s.dV;
        a.dt = cf.dt; a.kappa = cf.kappa;
        a.split = cf.split_orbit_at_knots;
        a.chunks = s.sw.chunks;
        a.nchunks = s.sw.nchunks;
        a.acc = s.acc;
        for (int d = 0; d < 3; ++d) a.scale[d] = s.scaleJ[d];
        a.stats = s.dstats;
        a.qtab = s.qtab;
        a.nq = s.nq;
        a.mnq = s.mnq;
        cudaEvent_t e0 = nullptr, e1 = nullptr;
        if (c->profiling) {
            UPIC_CUDA(c, cudaEventCreate(&e0));
            UPIC_CUDA(c, cudaEventCreate(&e1));
            UPIC_CUDA(c, cudaEventRecord(e0, c->st));
        }
        UPIC_CUDA(c, launch_implicit_map(s.order, s.uniform, a.split != 0, s.tg, a, s.grid, c->st, true));
        if (c->profiling) {
            UPIC_CUDA(c, cudaEventRecord(e1, c->st));
            c->prof_events.emplace_back(e0, e1);
        }
    }
    UPIC_CUDA(c, launch_convert_acc(s.acc, N, s.scaleJ, s.map, nullptr, 0.0, 1, c->st));
    // continuity, CN update of the potentials (:1474-1482)
    UPIC_CUDA(c, fft2d_batched(c->plan, s.Jhat, 3, 0, c->st, s.map));
    CnArgs k{};
    k.nx = c->nx; k.ny = c->ny; k.N = N;
    k.kx = c->d_kx; k.ky = c->d_ky; k.k2 = c->d_k2;
    k.excl = nullptr;
    k.Jhat = s.Jhat;
    k.st = s.spec;
    k.out = s.spec_out;
    k.gspec = s.gspec;
    k.dt = cf.dt; k.kappa = cf.kappa; k.sigma1 = cf.sigma1; k.sigma2 = cf.sigma2;
    UPIC_CUDA(c, launch_cn_kspace(k, c->st));
    UPIC_CUDA(c, fft2d_batched(c->plan, s.gspec, 2, 1, c->st, nullptr, 2, s.rec, kIRec, kIRecGpm));
    UPIC_CUDA(c, fft2d_batched(c->plan, s.gspec + 2 * (size_t)N, 3, 1, c->st, nullptr, 2, s.rec, kIRec, kIRecAe));
    // push (:1484-1505)
    PicardPushArgs q{};
    q.x = p.x; q.y = p.y; q.Px = p.Px; q.Py = p.Py; q.Pz = p.Pz; q.vx = p.vx; q.vy = p.vy; q.vz = p.vz;
    q.gx = s.gx; q.gy = s.gy; q.gz = s.gz;
    q.q = p.q; q.m = p.m; q.q0 = s.q0; q.m0 = s.m0;
    q.np = s.np;
    q.ox = o.x; q.oy = o.y; q.oPx = o.Px; q.oPy = o.Py; q.oPz = o.Pz; q.ovx = o.vx; q.ovy = o.vy; q.ovz = o.vz;
    q.nx = c->nx; q.ny = c->ny;
    q.Lx = cf.Lx; q.Ly = cf.Ly; q.inv_dx = 1.0 / s.dx; q.inv_dy = 1.0 / s.dy; q.dt = cf.dt;
    q.rec = s.rec;
    q.split = cf.split_orbit_at_knots;
    q.nq = s.nq;
    q.mnq = s.mnq;
    q.qtab = s.qtab;
    q.partials = s.partials;
    q.err = s.perr;
    UPIC_CUDA(c, launch_picard_push(s.order, s.uniform, q.split != 0, q, kNormGrid, s.dnorm, c->st));
    UPIC_CUDA(c, cudaMemcpyAsync(s.hstats, s.dstats, sizeof(MapStats), cudaMemcpyDeviceToHost, c->st));
    UPIC_CUDA(c, cudaMemcpyAsync(s.hnorm, s.dnorm, sizeof(NormSums), cudaMemcpyDeviceToHost, c->st));
    UPIC_CUDA(c, cudaMemcpyAsync(s.hflag, s.perr, sizeof(int), cudaMemcpyDeviceToHost, c->st));
    int rc = sync(c);
    if (rc) return rc;
    if (s.hstats->failures > 0 && (int)(s.hstats->first_fail_key & 0xffu) == kLocalNonfiniteIterate)
        return fail(c, UPIC_ERR_NONCONVERGED,
                    "Picard iterate velocity is not finite or exceeds 16 times the initial bound max(|v|, c)");
    if (s.hstats->failures > 0 || *s.hflag > 0)
        return fail(c, UPIC_ERR_TOO_LARGE, "an orbit crosses more spline knots than the kernel holds (38)");
    vel = *s.hnorm;
    return 0;
}

// One step of the non-relativistic method: picard_step_orbit
// (ec_pic_serial_demo.cpp:1509-1559).  The iteration count is a fixed upper
// limit; the reference accepts the last iterate when it is reached.
int picard_one_step(upic_ctx* c, ImplicitState& s, double* info) {
    const upic_config& cf = c->cfg;
    const int N = c->N, n3 = 3 * N;
    int rc;
    if (s.np > 0 && (rc = sort_active(c, s))) return rc;
    // A^n records for D_A and the start-point gathers
    UPIC_CUDA(c, cudaMemcpyAsync(s.dspec, s.spec + 3 * (size_t)N, sizeof(double2) * 3 * N,
                                 cudaMemcpyDeviceToDevice, c->st));
    UPIC_CUDA(c, fft2d_batched(c->plan, s.dspec, 3, 1, c->st, nullptr, 2, s.rec, kIRec, kIRecAn));
    const ParticleSoA& p = s.P[s.cur];
    const ParticleSoA& o = s.P[1 - s.cur];
    // v_guess = 2 v^n - v^{n-1} (:1514)
    if (s.np > 0) {
        UPIC_CUDA(c, launch_extrapolate((int)s.np, p.vx, p.wx, s.gx, c->st));
        UPIC_CUDA(c, launch_extrapolate((int)s.np, p.vy, p.wy, s.gy, c->st));
        UPIC_CUDA(c, launch_extrapolate((int)s.np, p.vz, p.wz, s.gz, c->st));
    }
    const size_t pb = sizeof(double) * s.np;
    auto guess_from_trial = [&]() -> int {
        if (s.np == 0) return 0;
        UPIC_CUDA(c, cudaMemcpyAsync(s.gx, o.vx, pb, cudaMemcpyDeviceToDevice, c->st));
        UPIC_CUDA(c, cudaMemcpyAsync(s.gy, o.vy, pb, cudaMemcpyDeviceToDevice, c->st));
        UPIC_CUDA(c, cudaMemcpyAsync(s.gz, o.vz, pb, cudaMemcpyDeviceToDevice, c->st));
        return 0;
    };
    bool have_prev = false, converged = false;
    int iters = 0;
    double cur_err = NAN, vel_err = NAN;
    for (int it = 0; it < cf.picard_max_iter; ++it) {
        NormSums vel;
        if ((rc = picard_eval(c, s, vel))) return rc;
        vel_err = relative_rms(vel, 3.0 * (double)s.np);
        cur_err = INFINITY;
        if (have_prev) {
            UPIC_CUDA(c, launch_residual_norms(N, s.map, s.Jprev, 1.0, 0.0, 1.0, s.partials, kNormGrid, s.dnorm,
                                               c->st));
            UPIC_CUDA(c, cudaMemcpyAsync(s.hnorm, s.dnorm, sizeof(NormSums), cudaMemcpyDeviceToHost, c->st));
            if ((rc = sync(c))) return rc;
            cur_err = relative_rms(*s.hnorm, (double)n3);
        }
        iters = it + 1;
        if (it > 0 && std::max(cur_err, vel_err) < cf.picard_tol) {
            converged = true;
            break;
        }
        UPIC_CUDA(c, cudaMemcpyAsync(s.Jprev, s.map, sizeof(double) * n3, cudaMemcpyDeviceToDevice, c->st));
        have_prev = true;
        if ((rc = guess_from_trial())) return rc;
    }
    if (cf.final_consistency_sweep) {
        // tr = evaluate_picard_map_orbit(tr.v_next, ...) (:1537-1539)
        if ((rc = guess_from_trial())) return rc;
        NormSums vel;
        if ((rc = picard_eval(c, s, vel))) return rc;
    }
    // accept: x, P, v from the trial set; v_prev = v^n; fields from spec_out
    ParticleSoA& nw = s.P[1 - s.cur];
    if (s.np > 0) {
        UPIC_CUDA(c, cudaMemcpyAsync(nw.wx, p.vx, pb, cudaMemcpyDeviceToDevice, c->st));
        UPIC_CUDA(c, cudaMemcpyAsync(nw.wy, p.vy, pb, cudaMemcpyDeviceToDevice, c->st));
        UPIC_CUDA(c, cudaMemcpyAsync(nw.wz, p.vz, pb, cudaMemcpyDeviceToDevice, c->st));
        UPIC_CUDA(c, cudaMemcpyAsync(nw.id, p.id, sizeof(int) * s.np, cudaMemcpyDeviceToDevice, c->st));
        if (!s.uniform) {
            UPIC_CUDA(c, cudaMemcpyAsync(nw.q, p.q, pb, cudaMemcpyDeviceToDevice, c->st));
            UPIC_CUDA(c, cudaMemcpyAsync(nw.m, p.m, pb, cudaMemcpyDeviceToDevice, c->st));
        }
    }
    s.cur = 1 - s.cur;
    std::swap(s.spec, s.spec_out);
    UPIC_CUDA(c, cudaMemcpyAsync(s.J, s.map, sizeof(double) * n3, cudaMemcpyDeviceToDevice, c->st));
    if (info) {
        for (int k = 0; k < UPIC_INFO_COUNT; ++k) info[k] = NAN;
        info[UPIC_INFO_ITERATIONS] = iters;
        info[UPIC_INFO_CONVERGED] = converged ? 1.0 : 0.0;
        info[UPIC_INFO_CURRENT_ERROR] = cur_err;
        info[UPIC_INFO_VELOCITY_ERROR] = vel_err;
        if ((rc = path_stats(c, s, info + UPIC_INFO_CROSSING_PARTICLES))) return rc;
    }
    ++s.steps;
    return sync(c);
}

// finite_node_vector (:5051) of a 3 x N node vector.
int all_finite(upic_ctx* c, ImplicitState& s, const double* v, bool& finite) {
    UPIC_CUDA(c, cudaMemsetAsync(s.dflag, 0, sizeof(int), c->st));
    UPIC_CUDA(c, launch_nonfinite_flag(3 * c->N, v, s.dflag, c->st));
    UPIC_CUDA(c, cudaMemcpyAsync(s.hflag, s.dflag, sizeof(int), cudaMemcpyDeviceToHost, c->st));
    const int rc = sync(c);
    if (rc) return rc;
    finite = *s.hflag == 0;
    return 0;
}

// nonlinear_residual_norms (:5576) on node vectors: the device sums and their
// copy to the host, queued on the context's stream ...
int launch_residual_sums(upic_ctx* c, ImplicitState& s, const double* map, const double* guess) {
    const upic_config& cf = c->cfg;
    const double floor_rel = 64.0 * DBL_EPSILON * cf.kappa;
    UPIC_CUDA(c, launch_residual_norms(c->N, map, guess, floor_rel, cf.nonlinear_atol, cf.nonlinear_rtol,
                                       s.partials, kNormGrid, s.dnorm, c->st));
    UPIC_CUDA(c, cudaMemcpyAsync(s.hnorm, s.dnorm, sizeof(NormSums), cudaMemcpyDeviceToHost, c->st));
    return 0;
}

// ... and the norms from the sums once the stream has reached them.
void norms_from_sums(upic_ctx* c, ImplicitState& s, Norms& n) {
    const upic_config& cf = c->cfg;
    const double floor_rel = 64.0 * DBL_EPSILON * cf.kappa;
    const double cnt = 3.0 * c->N;
    const NormSums& h = *s.hnorm;
    n.rms_absolute = std::sqrt((h.r2[0] + h.r2[1]) / cnt);
    const double map_rms = std::sqrt((h.map2[0] + h.map2[1]) / cnt);
    const double guess_rms = std::sqrt((h.guess2[0] + h.guess2[1]) / cnt);
    const double vrms = 0.5 * (map_rms + guess_rms);
    n.rms_relative = n.rms_absolute / (vrms + floor_rel);
    n.rms_scaled = n.rms_absolute / (cf.nonlinear_atol + cf.nonlinear_rtol * vrms);
    n.max_relative = h.max_rel;
    n.max_scaled = h.max_scaled;
}


// anderson_type2_candidate (:5763) over the last m+1 history entries.
int anderson_candidate(upic_ctx* c, ImplicitState& s, bool& ok) {
    const upic_config& cf = c->cfg;
    ok = false;
    const int available = s.hcount - 1;
    const int m = std::min(cf.anderson_memory, available);
    if (m <= 0) return 0;
    const int first = s.hcount - m - 1;
    const double* r[kHist];
    const double* x[kHist];
    for (int k = 0; k <= m; ++k) {
        r[k] = s.hr[first + k];
        x[k] = s.hx[first + k];
    }
    const int n3 = 3 * c->N;
    UPIC_CUDA(c, launch_anderson_dots(n3, r, m, s.partials, kNormGrid, s.ddots, c->st));
    const int ndots = m * (m + 1) / 2 + m;
    UPIC_CUDA(c, cudaMemcpyAsync(s.hdots, s.ddots, sizeof(double) * ndots, cudaMemcpyDeviceToHost, c->st));
    int rc = sync(c);
    if (rc) return rc;
    std::vector<std::vector<double>> gram(m, std::vector<double>(m, 0.0));
    std::vector<double> rhs(m, 0.0);
    int k = 0;
    for (int i = 0; i < m; ++i)
        for (int j = 0; j <= i; ++j) {
            gram[i][j] = gram[j][i] = s.hdots[k++];
        }
    double trace = 0.0;
    for (int i = 0; i < m; ++i) {
        rhs[i] = s.hdots[k++];
        trace += gram[i][i];
    }
    if (!(trace > 0.0) || !std::isfinite(trace)) return 0;
    std::vector<double> unreg;
    if (!solve_small_dense(gram, rhs, unreg)) return 0;
    const double regs = trace / (double)m;
    for (int i = 0; i < m; ++i) gram[i][i] += cf.anderson_regularization * regs;
    std::vector<double> gamma;
    if (!solve_small_dense(gram, rhs, gamma)) return 0;
    UPIC_CUDA(c, launch_anderson_candidate(n3, x, r, m, cf.anderson_damping, gamma.data(), s.cand, c->st));
    ok = true;
    return 0;
}

void push_history(upic_ctx* c, ImplicitState& s, const double* x, const double* r) {
    const int keep = c->cfg.anderson_memory + 1;
    if (s.hcount == keep) {
        double* tx = s.hx[0];
        double* tr = s.hr[0];
        for (int k = 0; k + 1 < s.hcount; ++k) {
            s.hx[k] = s.hx[k + 1];
            s.hr[k] = s.hr[k + 1];
        }
        s.hx[s.hcount - 1] = tx;
        s.hr[s.hcount - 1] = tr;
        --s.hcount;
    }
    const size_t bytes = sizeof(double) * 3 * (size_t)c->N;
    cudaMemcpyAsync(s.hx[s.hcount], x, bytes, cudaMemcpyDeviceToDevice, c->st);
    cudaMemcpyAsync(s.hr[s.hcount], r, bytes, cudaMemcpyDeviceToDevice, c->st);
    ++s.hcount;
}

void reset_history(upic_ctx* c, ImplicitState& s, const double* x, const double* r) {
    s.hcount = 0;
    push_history(c, s, x, r);
}

// The diagnostics row (compute_diagnostics :3521) of a state: its spectra
// and particle set (default: the current state).
int state_diagnostics(upic_ctx* c, ImplicitState& s, double* row, const double2* spec = nullptr, int pset = -1) {
    const upic_config& cf = c->cfg;
    const int N = c->N;
    if (!spec) spec = s.spec;
    if (pset < 0) pset = s.cur;
    UPIC_CUDA(c, launch_diag_spectra(N, c->d_kx, c->d_ky, spec, s.dspec, c->st));
    // mode amplitudes from the spectra before the inverse transforms overwrite them
    const int mode = cf.perturbation_mode;
    const int im = ((mode % c->nx) + c->nx) % c->nx, jm = ((mode % c->ny) + c->ny) % c->ny;
    const int idx = im * c->ny, idy = jm;
    double2 modes[3];
    UPIC_CUDA(c, cudaMemcpyAsync(&modes[0], spec + 2 * (size_t)N + idx, sizeof(double2), cudaMemcpyDeviceToHost, c->st));
    UPIC_CUDA(c, cudaMemcpyAsync(&modes[1], s.dspec + idx, sizeof(double2), cudaMemcpyDeviceToHost, c->st));
    UPIC_CUDA(c, cudaMemcpyAsync(&modes[2], s.dspec + 5 * (size_t)N + idy, sizeof(double2), cudaMemcpyDeviceToHost, c->st));
    UPIC_CUDA(c, fft2d_batched(c->plan, s.dspec, 10, 1, c->st, nullptr, 1, s.dreal));
    ImplicitDiagArgs d{};
    d.N = N;
    d.E = s.dreal;
    d.B = s.dreal + 3 * (size_t)N;
    d.divE = s.dreal + 6 * (size_t)N;
    d.divA = s.dreal + 7 * (size_t)N;
    d.psi = s.dreal + 8 * (size_t)N;
    d.rho = s.dreal + 9 * (size_t)N;
    d.sigma1 = cf.sigma1;
    d.kappa = cf.kappa;
    d.partials = s.partials;
    d.grid = kNormGrid;
    UPIC_CUDA(c, launch_implicit_diag(d, s.ddots, c->st));
    const ParticleSoA& p = s.P[pset];
    UPIC_CUDA(c, launch_kinetic(s.np, p.vx, p.vy, p.vz, s.uniform ? nullptr : p.m, s.m0, cf.kappa,
                                s.partials + 32 * kNormGrid, kNormGrid, s.ddots + 20, c->st, s.picard));
    UPIC_CUDA(c, cudaMemcpyAsync(s.hdots, s.ddots, sizeof(double) * 22, cudaMemcpyDeviceToHost, c->st));
    int rc = sync(c);
    if (rc) return rc;
    const double* h = s.hdots;
    const double invN = 1.0 / N;
    auto tot = [&](int k) { return h[2 * k] + h[2 * k + 1]; };
    auto rel = [](double a, double b) { return b > 0.0 ? a / b : (a == 0.0 ? 0.0 : INFINITY); };
    double* r = row;
    r[UPIC_P3_GAUSS_RMS] = std::sqrt(tot(0) * invN);
    r[UPIC_P3_GAUSS_MAX] = h[18];
    r[UPIC_P3_DIVE_RMS] = std::sqrt(tot(1) * invN);
    r[UPIC_P3_SIGMA1_RHO_RMS] = std::fabs(cf.sigma1) * std::sqrt(tot(2) * invN);
    r[UPIC_P3_GAUSS_NORM_RMS] = r[UPIC_P3_DIVE_RMS] + r[UPIC_P3_SIGMA1_RHO_RMS];
    r[UPIC_P3_GAUSS_RELATIVE] = rel(r[UPIC_P3_GAUSS_RMS], r[UPIC_P3_GAUSS_NORM_RMS]);
    r[UPIC_P3_GAUGE_RMS] = std::sqrt(tot(3) * invN);
    r[UPIC_P3_GAUGE_MAX] = h[19];
    r[UPIC_P3_PSI_OVER_KAPPA2_RMS] = std::sqrt(tot(4) * invN) / (cf.kappa * cf.kappa);
    r[UPIC_P3_DIVA_RMS] = std::sqrt(tot(5) * invN);
    r[UPIC_P3_GAUGE_NORM_RMS] = r[UPIC_P3_PSI_OVER_KAPPA2_RMS] + r[UPIC_P3_DIVA_RMS];
    r[UPIC_P3_GAUGE_RELATIVE] = rel(r[UPIC_P3_GAUGE_RMS], r[UPIC_P3_GAUGE_NORM_RMS]);
    r[UPIC_P3_FIELD_ENERGY] = (0.5 / cf.sigma1 * tot(6) + 0.5 / cf.sigma2 * tot(7)) * s.dV;
    r[UPIC_P3_KINETIC_ENERGY] = h[20] + h[21];
    r[UPIC_P3_TOTAL_ENERGY] = r[UPIC_P3_FIELD_ENERGY] + r[UPIC_P3_KINETIC_ENERGY];
    r[UPIC_P3_RHO_MODE] = std::hypot(modes[0].x, modes[0].y) * invN;
    r[UPIC_P3_E_MODE_RE] = modes[1].x * invN;
    r[UPIC_P3_E_MODE_IM] = modes[1].y * invN;
    r[UPIC_P3_E_MODE_ABS] = std::hypot(modes[1].x, modes[1].y) * invN;
    r[UPIC_P3_BZ_Y_MODE_RE] = modes[2].x * invN;
    r[UPIC_P3_BZ_Y_MODE_IM] = modes[2].y * invN;
    r[UPIC_P3_BZ_Y_MODE_ABS] = std::hypot(modes[2].x, modes[2].y) * invN;
    r[UPIC_P3_MEAN_RHO] = tot(8) / (double)N;
    return 0;
}

// Knot-crossing statistics of the step just accepted (the orbits from the
// spare set's positions): crossing particles, average and maximum segments
// per orbit (PathStats, ec_pic_nyquist_projected.cpp and
// ec_pic_serial_demo.cpp:835).  Orbit velocity: the stored vbar, or for the
// Picard method (v^{n+1} + v^n) / 2 as Project1's main loop forms it.
int path_stats(upic_ctx* c, ImplicitState& s, double* out3) {
    const upic_config& cf = c->cfg;
    const ParticleSoA& p0 = s.P[1 - s.cur];
    const ParticleSoA& p1 = s.P[s.cur];
    PathStatsArgs a{};
    a.x = p0.x;
    a.y = p0.y;
    if (s.picard) {
        a.v1x = p1.vx;
        a.v1y = p1.vy;
        a.v0x = p0.vx;
        a.v0y = p0.vy;
    } else {
        a.bx = s.bx[s.cur];
        a.by = s.by[s.cur];
    }
    a.np = s.np;
    a.nx = c->nx;
    a.ny = c->ny;
    a.Lx = cf.Lx;
    a.Ly = cf.Ly;
    a.dt = cf.dt;
    a.split = cf.split_orbit_at_knots;
    a.counts = s.pstat;
    unsigned long long h[4];
    UPIC_CUDA(c, cudaMemsetAsync(s.pstat, 0, sizeof(unsigned long long) * 4, c->st));
    if (s.np > 0) UPIC_CUDA(c, launch_path_stats(s.order, a, c->st));
    UPIC_CUDA(c, cudaMemcpyAsync(h, s.pstat, sizeof(h), cudaMemcpyDeviceToHost, c->st));
    const int rc = sync(c);
    if (rc) return rc;
    out3[0] = (double)h[2];
    out3[1] = s.np ? (double)h[0] / (double)s.np : (s.picard ? 0.0 : 1.0);
    out3[2] = (double)(s.np ? h[3] : 1);
    return 0;
}

// One implicit step (nonlinear_step_uniform_subcycled :5878); info: the
// UPIC_INFO_* entries.
// Result of one outer current solve (from the first guess to the accepted
// final evaluation).
struct OuterResult {
    int iterations = 0, anderson_steps = 0, picard_steps = 0;
    int restarts = 0, backtracked = 0, method = UPIC_METHOD_CODE_NONE;
    double min_alpha = 1.0, observed_rate = INFINITY, contraction = INFINITY;
    Norms fin;
    MapStats ms{};
};

// The outer current iteration of nonlinear_step_uniform_subcycled (:5878) at
// the current particle layout: first guess, Anderson / damped Picard updates
// with backtracking, the final consistency evaluation (:6160) that writes the
// trial state.  Returns UPIC_ERR_LOCAL_PARTICLE when a local particle solve
// fails in any evaluation (SelectiveParticleRefinementNeeded).
int outer_solve(upic_ctx* c, ImplicitState& s, OuterResult& out) {
    const upic_config& cf = c->cfg;
    const int N = c->N, n3 = 3 * N;
    int rc;
    out = OuterResult{};
    s.warm_valid = false;
    UPIC_CUDA(c, cudaMemcpyAsync(s.guess, s.J0, sizeof(double) * n3, cudaMemcpyDeviceToDevice, c->st));
    bool finite = true;
    if ((rc = all_finite(c, s, s.guess, finite))) return rc;
    if (!finite) return fail(c, UPIC_ERR_NONFINITE, "nonfinite initial macro-current predictor");
    const bool anderson = cf.nonlinear_solver == UPIC_SOLVER_ANDERSON;
    s.hcount = 0;
    s.map_eval = 0;
    double prev_rms = INFINITY, first_rms = INFINITY;
    bool have_prefetched = false, converged = false;
    int iterations = 0, anderson_steps = 0, picard_steps = 0, restarts = 0, backtracked = 0;
    double min_alpha = 1.0;
    // update_method of the last accepted update (:5902-5903, :6122-6128)
    int method = anderson ? UPIC_METHOD_CODE_PICARD_FALLBACK : UPIC_METHOD_CODE_PICARD;
    Norms norms, prefetched_norms;
    MapStats ms{};
    for (int it = 0; it < cf.nonlinear_max_iter; ++it) {
        if (!have_prefetched) {
            if ((rc = eval_map(c, s, s.guess, s.map, false, &ms, &finite, &norms))) {
                out.iterations = it + 1;  // the iterations a failed attempt reports (:5949-5953)
                return rc;
            }
            if (!finite)
                return fail(c, UPIC_ERR_NONCONVERGED, "uniform particle map returned a nonfinite macro current");
        } else {
            norms = prefetched_norms;  // the accepted trial's norms: the same (map, guess) pair
            // secant contraction against the previous iterate, which the
            // swap after the accepted update left in trial / trial_map
            // (:5981-5996); read back with the final evaluation
            const double* xs[2] = {s.trial, s.guess};
            const double* gs[2] = {s.trial_map, s.map};
            UPIC_CUDA(c, launch_anderson_dots(n3, xs, 1, s.partials, kNormGrid, s.dcon + 4 * (size_t)it, c->st));
            UPIC_CUDA(c, launch_anderson_dots(n3, gs, 1, s.partials, kNormGrid, s.dcon + 4 * (size_t)it + 2,
                                              c->st));
        }
        have_prefetched = false;
        UPIC_CUDA(c, launch_axpy(n3, s.map, s.guess, -1.0, s.resid, c->st));
        iterations = it + 1;
        if (it == 0) first_rms = norms.rms_relative;
        if (norms.rms_scaled <= 1.0 && norms.max_scaled <= 1.0) {
            converged = true;
            break;
        }
        if (anderson && std::isfinite(prev_rms) && norms.rms_relative > cf.anderson_growth_limit * prev_rms) {
            s.hcount = 0;
            ++restarts;
        }
        push_history(c, s, s.guess, s.resid);
        bool used_anderson = false;
        if (anderson && it >= cf.anderson_start && s.hcount >= 2) {
            if ((rc = anderson_candidate(c, s, used_anderson))) return rc;
            if (used_anderson) {
                if ((rc = all_finite(c, s, s.cand, finite))) return rc;
                used_anderson = finite;
            }
            if (!used_anderson) {
                reset_history(c, s, s.guess, s.resid);
                ++restarts;
            }
        }
        const double cur_rms = norms.rms_scaled, cur_max = norms.max_scaled;
        // backtracking line search on the candidate (:6044-6084)
        // cand_finite: the candidate is known to be finite, and so is every
        // trial between it and the (finite) current guess
        double accepted_alpha = 1.0;
        auto try_update = [&](bool& accepted, bool cand_finite) -> int {
            accepted = false;
            for (int bt = 0; bt <= 6; ++bt) {
                const double alpha = std::ldexp(1.0, -bt);
                accepted_alpha = alpha;
                UPIC_CUDA(c, launch_lerp(n3, s.guess, s.cand, alpha, s.trial, c->st));
                int r2;
                if (!cand_finite) {
                    bool tf = true;
                    if ((r2 = all_finite(c, s, s.trial, tf))) return r2;
                    if (!tf) continue;
                }
                Norms tn;
                r2 = eval_map(c, s, s.trial, s.trial_map, false, &ms, nullptr, &tn);
                if (r2) return r2;
                if (!std::isfinite(tn.rms_scaled)) continue;
                const bool dec = tn.rms_scaled <= (1.0 - 1.0e-4 * alpha) * cur_rms;
                const bool safe = tn.max_scaled <= cf.anderson_growth_limit * cur_max;
                if (dec && safe) {
                    prefetched_norms = tn;
                    accepted = true;
                    return 0;
                }
            }
            return 0;
        };
        bool accepted = false, as_anderson = false;
        if (used_anderson) {
            if ((rc = try_update(accepted, true))) return rc;
            as_anderson = accepted;
            if (!accepted) {
                reset_history(c, s, s.guess, s.resid);
                ++restarts;
            }
        }
        if (!accepted) {
            const double damping = anderson ? cf.anderson_damping : 1.0;
            UPIC_CUDA(c, launch_axpy(n3, s.guess, s.resid, damping, s.cand, c->st));
            if ((rc = try_update(accepted, false))) return rc;
        }
        if (!accepted)
            return fail(c, UPIC_ERR_NONCONVERGED,
                        "outer current Anderson/Picard backtracking failed at the prescribed macro dt");
        if (as_anderson) ++anderson_steps;
        else ++picard_steps;
        const bool bt = accepted_alpha < 1.0;
        method = as_anderson ? (bt ? UPIC_METHOD_CODE_ANDERSON_BACKTRACKED : UPIC_METHOD_CODE_ANDERSON)
                             : (bt ? UPIC_METHOD_CODE_CURRENT_PICARD_BACKTRACKED : UPIC_METHOD_CODE_CURRENT_PICARD);
        if (bt) {
            ++backtracked;
            min_alpha = std::min(min_alpha, accepted_alpha);
        }
        prev_rms = norms.rms_relative;
        std::swap(s.guess, s.trial);
        std::swap(s.map, s.trial_map);
        have_prefetched = true;
    }
    if (!converged) {
        char buf[160];
        std::snprintf(buf, sizeof(buf), "outer macro-current solve failed at dt=%g after %d iterations", cf.dt,
                      iterations);
        return fail(c, UPIC_ERR_NONCONVERGED, buf);
    }
    // the contraction sums of iterations 1.., read with the final evaluation
    if (iterations > 1)
        UPIC_CUDA(c, cudaMemcpyAsync(s.hcon, s.dcon, sizeof(double) * 4 * (size_t)iterations, cudaMemcpyDeviceToHost,
                                     c->st));
    // final consistency evaluation (:6160) produces the accepted state
    Norms fin;
    if ((rc = eval_map(c, s, s.guess, s.map, true, &ms, nullptr, &fin))) return rc;
    if (!(fin.rms_scaled <= 1.0 && fin.max_scaled <= 1.0))
        return fail(c, UPIC_ERR_NONCONVERGED,
                    "final outer macro-current consistency evaluation failed at the prescribed macro dt");
    out.iterations = iterations;
    out.anderson_steps = anderson_steps;
    out.picard_steps = picard_steps;
    out.restarts = restarts;
    out.backtracked = backtracked;
    out.min_alpha = min_alpha;
    out.method = method;
    out.contraction = INFINITY;
    for (int it = 1; it < iterations; ++it) {
        const double dx2 = s.hcon[4 * it], dg2 = s.hcon[4 * it + 2];
        const double dx_rms = std::sqrt(dx2 / (double)n3);
        if (dx_rms > 64.0 * DBL_EPSILON) out.contraction = std::sqrt(dg2 / (double)n3) / dx_rms;
    }
    // observed_nonlinear_convergence_rate (:5534): one history entry per
    // outer iteration, the first holding the first relative rms residual
    out.observed_rate = INFINITY;
    if (iterations >= 2 && first_rms > 0.0 && fin.rms_relative >= 0.0 && std::isfinite(fin.rms_relative)) {
        if (fin.rms_relative == 0.0) {
            out.observed_rate = 0.0;
        } else {
            const double ratio = fin.rms_relative / first_rms;
            if (ratio > 0.0 && std::isfinite(ratio)) out.observed_rate = std::pow(ratio, 1.0 / (double)(iterations - 1));
        }
    }
    out.fin = fin;
    out.ms = ms;
    return 0;
}

// Upload the particle layout (substeps per sorted particle), the compact
// list of refined particles and their sub-orbit record offsets; grow the
// sub-orbit record buffer to the refined particles' substeps.
int upload_layout(upic_ctx* c, ImplicitState& s) {
    std::vector<int> refined, roff;
    long total = 0, rtotal = 0;
    for (long p = 0; p < s.np; ++p) {
        total += s.h_nsub[p];
        if (s.h_nsub[p] > 1) {
            refined.push_back((int)p);
            roff.push_back((int)rtotal);
            rtotal += s.h_nsub[p];
        }
    }
    s.nref = (int)refined.size();
    s.total_substeps = total;
    if (rtotal > s.sub_cap) {
        int rc;
        if ((rc = sync(c))) return rc;
        dfree(c, s.sub_rec);
        s.sub_rec = nullptr;
        s.sub_cap = 0;
        if ((rc = dalloc(c, &s.sub_rec, 5 * (size_t)rtotal))) return rc;
        s.sub_cap = rtotal;
    }
    UPIC_CUDA(c, cudaMemcpyAsync(s.nsub, s.h_nsub.data(), sizeof(int) * s.np, cudaMemcpyHostToDevice, c->st));
    if (s.nref > 0) {
        UPIC_CUDA(c, cudaMemcpyAsync(s.refined, refined.data(), sizeof(int) * s.nref, cudaMemcpyHostToDevice, c->st));
        UPIC_CUDA(c, cudaMemcpyAsync(s.roff, roff.data(), sizeof(int) * s.nref, cudaMemcpyHostToDevice, c->st));
    }
    return sync(c);
}

// Append the accepted state's J, A and phi to the learned predictor's
// frames (A and phi transformed back from the state spectra).
int push_frame(upic_ctx* c, ImplicitState& s) {
    const size_t N = (size_t)c->N;
    UPIC_CUDA(c, cudaMemcpyAsync(s.dspec, s.spec + 3 * N, sizeof(double2) * 3 * N, cudaMemcpyDeviceToDevice, c->st));
    UPIC_CUDA(c, fft2d_batched(c->plan, s.dspec, 3, 1, c->st, nullptr, 1, s.fbuf));
    UPIC_CUDA(c, cudaMemcpyAsync(s.dspec, s.spec, sizeof(double2) * N, cudaMemcpyDeviceToDevice, c->st));
    UPIC_CUDA(c, fft2d_batched(c->plan, s.dspec, 1, 1, c->st, nullptr, 1, s.fbuf + 3 * N));
    UPIC_CUDA(c, gnet::net_push_frame(s.net, s.J, s.fbuf, s.fbuf + 3 * N, c->st));
    return 0;
}

// First guess J0 of this step's outer current iteration (UPIC_PREDICTOR_*),
// with the extrapolation Jx and the learned prediction Jl it was chosen from.
int form_guess(upic_ctx* c, ImplicitState& s) {
    const upic_config& cf = c->cfg;
    const int n3 = 3 * c->N;
    s.have_Jx = s.have_Jl = false;
    if (cf.current_predictor == UPIC_PREDICTOR_EXTRAPOLATED && s.have_Jold) {
        UPIC_CUDA(c, launch_extrapolate(n3, s.J, s.Jold, s.Jx, c->st));
        s.have_Jx = true;
    } else if (cf.current_predictor == UPIC_PREDICTOR_LEARNED && gnet::net_frames(s.net) >= 2) {
        UPIC_CUDA(c, gnet::net_extrapolate(s.net, s.Jx, c->st));
        s.have_Jx = true;
        if (gnet::net_frames(s.net) >= gnet::kFrames && s.trained_steps > 0) {
            UPIC_CUDA(c, gnet::net_predict(s.net, s.Jl, c->st));
            s.have_Jl = true;
        }
    }
    const double* g = s.J;
    s.predictor_used = UPIC_PREDICTOR_PREVIOUS;
    if (s.have_Jl && s.use_learned) {
        g = s.Jl;
        s.predictor_used = UPIC_PREDICTOR_LEARNED;
    } else if (s.have_Jx) {
        g = s.Jx;
        s.predictor_used = UPIC_PREDICTOR_EXTRAPOLATED;
    }
    UPIC_CUDA(c, cudaMemcpyAsync(s.J0, g, sizeof(double) * n3, cudaMemcpyDeviceToDevice, c->st));
    return 0;
}

// After the accepted current J^{n+1} is in s.J: distances of the guess, the
// extrapolation and the learned prediction from it (into info), and for the
// learned predictor the choice of the next step's guess, a training step on
// this step's sample and the new frame.
int predictor_update(upic_ctx* c, ImplicitState& s, double* info) {
    const upic_config& cf = c->cfg;
    const int N = c->N;
    const bool learned = cf.current_predictor == UPIC_PREDICTOR_LEARNED;
    if (!info && !learned) return 0;
    const double* cand[3] = {s.J0, s.have_Jx ? s.Jx : nullptr, s.have_Jl ? s.Jl : nullptr};
    for (int k = 0; k < 3; ++k)
        if (cand[k])
            UPIC_CUDA(c, launch_residual_norms(N, s.J, cand[k], 1.0, 0.0, 1.0, s.partials, kNormGrid, s.dnorm3 + k,
                                               c->st));
    bool trained = false;
    if (learned && gnet::net_frames(s.net) >= gnet::kFrames && s.trained_steps < cf.learned_train_steps) {
        UPIC_CUDA(c, gnet::net_train(s.net, s.J, cf.learned_train_iters, (float)cf.learned_rate, s.dloss, c->st));
        ++s.trained_steps;
        trained = true;
    }
    UPIC_CUDA(c, cudaMemcpyAsync(s.hnorm3, s.dnorm3, sizeof(NormSums) * 3, cudaMemcpyDeviceToHost, c->st));
    if (trained) UPIC_CUDA(c, cudaMemcpyAsync(s.hloss, s.dloss, sizeof(double), cudaMemcpyDeviceToHost, c->st));
    int rc;
    if (learned && (rc = push_frame(c, s))) return rc;
    int nerr = 0;
    if (learned) UPIC_CUDA(c, cudaMemcpyAsync(&nerr, gnet::net_error_flag(s.net), sizeof(int), cudaMemcpyDeviceToHost,
                                              c->st));
    if ((rc = sync(c))) return rc;
    if (nerr) return fail(c, UPIC_ERR_CUDA, "learned predictor: a tensor-core wait timed out");
    double err[3] = {NAN, NAN, NAN};
    for (int k = 0; k < 3; ++k)
        if (cand[k]) {
            const NormSums& h = s.hnorm3[k];
            const double m2 = h.map2[0] + h.map2[1];
            err[k] = std::sqrt((h.r2[0] + h.r2[1]) / (m2 > 0.0 ? m2 : 1.0e-300));
        }
    if (learned) s.use_learned = s.have_Jl && s.have_Jx && err[2] < err[1];
    if (info) {
        info[UPIC_INFO_PREDICTOR_USED] = s.predictor_used;
        info[UPIC_INFO_GUESS_ERROR] = err[0];
        info[UPIC_INFO_EXTRAPOLATION_ERROR] = err[1];
        info[UPIC_INFO_LEARNED_ERROR] = err[2];
        info[UPIC_INFO_LEARNED_LOSS] = trained ? *s.hloss : NAN;
    }
    return 0;
}

// One implicit step (nonlinear_step_orbit :6477): the full-dt solve, and when
// a local particle solve fails and selective_particle_fallback is set, the
// selective sub-cycling fallback (nonlinear_step_selective_particle_fallback
// :6328): every failing particle's substep count doubles (up to
// selective_particle_max_substeps) and the outer solve restarts from its
// first guess, until it succeeds.
int implicit_one_step(upic_ctx* c, ImplicitState& s, double* info) {
    const upic_config& cf = c->cfg;
    const int N = c->N, n3 = 3 * N;
    int rc;
    if (s.np > 0 && (rc = sort_active(c, s))) return rc;
    // A^n records for the orbit D_A and the start-point gather
    UPIC_CUDA(c, cudaMemcpyAsync(s.dspec, s.spec + 3 * (size_t)N, sizeof(double2) * 3 * N,
                                 cudaMemcpyDeviceToDevice, c->st));
    UPIC_CUDA(c, fft2d_batched(c->plan, s.dspec, 3, 1, c->st, nullptr, 2, s.rec, kIRec, kIRecAn));
    s.layout_active = false;
    s.nref = 0;
    s.total_substeps = s.np;
    if ((rc = form_guess(c, s))) return rc;
    OuterResult r;
    rc = outer_solve(c, s, r);
    int restarts = 0, direct_iterations = 0;
    bool fallback_used = false;
    if (rc == UPIC_ERR_LOCAL_PARTICLE && cf.selective_particle_fallback && s.np > 0) {
        fallback_used = true;
        direct_iterations = r.iterations;
        const std::string direct = c->err;
        s.h_nsub.assign(s.np, 1);
        if ((rc = upload_layout(c, s))) return rc;
        s.layout_active = true;
        for (;;) {
            s.layout_restart = restarts;
            rc = outer_solve(c, s, r);
            if (rc != UPIC_ERR_LOCAL_PARTICLE) break;
            int nf = 0;
            UPIC_CUDA(c, cudaMemcpy(&nf, s.nfailed, sizeof(int), cudaMemcpyDeviceToHost));
            std::vector<int> failed(nf);
            if (nf > 0)
                UPIC_CUDA(c, cudaMemcpy(failed.data(), s.failed, sizeof(int) * nf, cudaMemcpyDeviceToHost));
            long exhausted = 0;
            for (int p : failed)
                if (s.h_nsub[p] >= cf.selective_particle_max_substeps) ++exhausted;
            if (exhausted > 0)
                for (size_t k = s.fail_event; k < s.faillog.size(); k += UPIC_FAILLOG_COUNT)
                    s.faillog[k + UPIC_FAILLOG_EXHAUSTED] = 1.0;
            if (exhausted > 0) {
                char buf[400];
                std::snprintf(buf, sizeof(buf),
                              "direct macro solve failed (%s); selective particle fallback reached h=dt/%d with %ld "
                              "particles still unconverged; macro dt=%g was not changed",
                              direct.c_str(), cf.selective_particle_max_substeps, exhausted, cf.dt);
                rc = fail(c, UPIC_ERR_NONCONVERGED, buf);
                break;
            }
            for (int p : failed) s.h_nsub[p] = std::min(cf.selective_particle_max_substeps, 2 * s.h_nsub[p]);
            ++restarts;
            if ((rc = upload_layout(c, s))) return rc;
        }
        s.layout_active = false;
        if (rc == UPIC_ERR_NONCONVERGED && c->err.find("selective particle fallback") == std::string::npos) {
            const std::string inner = c->err;
            rc = fail(c, UPIC_ERR_NONCONVERGED,
                      "direct macro solve failed (" + direct +
                          "); selective outer current solve also failed without a refinable local-particle set (" +
                          inner + ")");
        }
    }
    if (rc == UPIC_ERR_LOCAL_PARTICLE && !cf.selective_particle_fallback) {
        // write_failed_particle_diagnostics(..., 0, cfg, failures, true) (:6514)
        for (size_t k = s.fail_event; k < s.faillog.size(); k += UPIC_FAILLOG_COUNT) {
            s.faillog[k + UPIC_FAILLOG_RESTART] = 0.0;
            s.faillog[k + UPIC_FAILLOG_EXHAUSTED] = 1.0;
        }
    }
    if (rc) return rc;
    s.last_refined = s.nref;
    const int iterations = r.iterations, anderson_steps = r.anderson_steps, picard_steps = r.picard_steps;
    const Norms& fin = r.fin;
    const MapStats& ms = r.ms;
    // accept: particles from the trial set, v_prev = v^n, fields from the trial spectra
    ParticleSoA& old = s.P[s.cur];
    ParticleSoA& nw = s.P[1 - s.cur];
    const size_t pb = sizeof(double) * s.np;
    if (s.np > 0) {
        UPIC_CUDA(c, cudaMemcpyAsync(nw.wx, old.vx, pb, cudaMemcpyDeviceToDevice, c->st));
        UPIC_CUDA(c, cudaMemcpyAsync(nw.wy, old.vy, pb, cudaMemcpyDeviceToDevice, c->st));
        UPIC_CUDA(c, cudaMemcpyAsync(nw.wz, old.vz, pb, cudaMemcpyDeviceToDevice, c->st));
        UPIC_CUDA(c, cudaMemcpyAsync(nw.id, old.id, sizeof(int) * s.np, cudaMemcpyDeviceToDevice, c->st));
        if (!s.uniform) {
            UPIC_CUDA(c, cudaMemcpyAsync(nw.q, old.q, pb, cudaMemcpyDeviceToDevice, c->st));
            UPIC_CUDA(c, cudaMemcpyAsync(nw.m, old.m, pb, cudaMemcpyDeviceToDevice, c->st));
        }
    }
    s.cur = 1 - s.cur;
    std::swap(s.spec, s.spec_out);
    if (cf.current_predictor == UPIC_PREDICTOR_EXTRAPOLATED) {
        UPIC_CUDA(c, cudaMemcpyAsync(s.Jold, s.J, sizeof(double) * n3, cudaMemcpyDeviceToDevice, c->st));
        s.have_Jold = true;
    }
    UPIC_CUDA(c, cudaMemcpyAsync(s.J, s.map, sizeof(double) * n3, cudaMemcpyDeviceToDevice, c->st));
    if (info) {
        info[UPIC_INFO_ITERATIONS] = iterations;
        info[UPIC_INFO_CONVERGED] = 1.0;
        info[UPIC_INFO_FINAL_RMS_RESIDUAL] = fin.rms_relative;
        info[UPIC_INFO_FINAL_MAX_PARTICLE_RESIDUAL] = fin.max_relative;
        info[UPIC_INFO_LOCAL_ITER_MAX] = ms.iter_max;
        info[UPIC_INFO_LOCAL_ITER_MEAN] = s.np > 0 ? (double)ms.iter_total / (double)s.total_substeps : 0.0;
        info[UPIC_INFO_ANDERSON_STEPS] = anderson_steps;
        info[UPIC_INFO_PICARD_STEPS] = picard_steps;
        info[UPIC_INFO_CURRENT_ERROR] = NAN;
        info[UPIC_INFO_VELOCITY_ERROR] = NAN;
        int rc2 = path_stats(c, s, info + UPIC_INFO_CROSSING_PARTICLES);
        if (rc2) return rc2;
        info[UPIC_INFO_SELECTIVE_FALLBACK_USED] = fallback_used ? 1.0 : 0.0;
        info[UPIC_INFO_SELECTIVE_RESTARTS] = restarts;
        info[UPIC_INFO_SELECTIVE_REFINED] = s.nref;
        info[UPIC_INFO_SELECTIVE_SUBSTEPS] = (double)s.total_substeps;
        info[UPIC_INFO_ANDERSON_RESTARTS] = r.restarts;
        info[UPIC_INFO_FINAL_ABS_RMS_RESIDUAL] = fin.rms_absolute;
        info[UPIC_INFO_OBSERVED_RATE] = r.observed_rate;
        info[UPIC_INFO_MAP_CONTRACTION] = r.contraction;
        info[UPIC_INFO_BACKTRACKED_STEPS] = r.backtracked;
        info[UPIC_INFO_MIN_UPDATE_ALPHA] = r.min_alpha;
        info[UPIC_INFO_CONVERGENCE_METHOD] =
            r.method + (fallback_used ? UPIC_METHOD_FORM_SELECTIVE : UPIC_METHOD_FORM_DIRECT);
        info[UPIC_INFO_DIRECT_ATTEMPT_ITERATIONS] = fallback_used ? direct_iterations : 0;
        // the particle layout: 1 substep each unless the fallback refined it
        long counts[7] = {0, 0, 0, 0, 0, 0, 0};
        int max_sub = 1;
        if (fallback_used) {
            for (int n : s.h_nsub) {
                int level = 0;
                for (int v = n; v > 1; v /= 2) ++level;
                ++counts[std::min(level, 6)];
                max_sub = std::max(max_sub, n);
            }
        } else {
            counts[0] = s.np;
        }
        info[UPIC_INFO_SUBSTEPS_USED] = s.np > 0 ? max_sub : 0;
        info[UPIC_INFO_SELECTIVE_WORK_RATIO] = s.np > 0 ? (double)s.total_substeps / (double)s.np : 0.0;
        for (int k = 0; k < 7; ++k) info[UPIC_INFO_SELECTIVE_N1 + k] = (double)counts[k];
    }
    if ((rc = predictor_update(c, s, info))) return rc;
    ++s.steps;
    return sync(c);
}

// wrap1 of positions outside [-L/2, L/2); positions inside are kept as
// given (a second wrap of a wrapped value can move it by an ulp).
__global__ void wrap_positions_kernel(double* x, double* y, long n, double Lx, double Ly) {
    for (long p = blockIdx.x * (long)blockDim.x + threadIdx.x; p < n; p += (long)gridDim.x * blockDim.x) {
        if (!(x[p] >= -0.5 * Lx && x[p] < 0.5 * Lx)) {
            double a = fmod(x[p] + 0.5 * Lx, Lx);
            if (a < 0.0) a += Lx;
            x[p] = a - 0.5 * Lx;
        }
        if (!(y[p] >= -0.5 * Ly && y[p] < 0.5 * Ly)) {
            double b = fmod(y[p] + 0.5 * Ly, Ly);
            if (b < 0.0) b += Ly;
            y[p] = b - 0.5 * Ly;
        }
    }
}

}  // namespace

// ---------------------------------------------------------------------------
int implicit_create(upic_ctx* c) {
    auto* s = new ImplicitState();
    c->imp = s;
    if (c->cfg.method == UPIC_METHOD_CN_ORBIT_NONREL) {
        // Project1's constants in the roles of Project3's: light speed c,
        // scalar source 1/eps0, vector source mu0; no Nyquist projection
        c->cfg.kappa = c->cfg.c;
        c->cfg.sigma1 = 1.0 / c->cfg.eps0;
        c->cfg.sigma2 = c->cfg.mu0;
        c->cfg.nyquist_projection = 0;
        s->picard = true;
    }
    const upic_config& cf = c->cfg;
    s->order = cf.spline_order;
    s->nq = cf.orbit_quad_order;
    s->dx = cf.Lx / c->nx;
    s->dy = cf.Ly / c->ny;
    s->dV = s->dx * s->dy * cf.Lz;
    const int N = c->N;
    // window guard: the orbit reaches kappa*dt from its start; sorting every
    // step leaves no drift on top of that
    const double reach = cf.kappa * cf.dt / std::min(s->dx, s->dy);
    s->dt_max = cf.dt;
    const int guard = cf.guard >= 0 ? cf.guard : (s->picard ? 2 : (int)std::ceil(reach) + 1);
    const int tile = cf.tile > 0 ? cf.tile : 8;
    s->tg = make_tiles(c->nx, c->ny, tile, guard, s->order / 2, s->order / 2 + 1);
    s->tg.key_origin_x = 0.5 * cf.Lx;
    s->tg.key_origin_y = 0.5 * cf.Ly;
    s->tg.key_shift = 0.0;
    s->tg.chunk = kMaxImplicitChunk;
    const bool split = cf.split_orbit_at_knots != 0;
    if (implicit_configure_smem(s->tg, s->order, split, s->picard) != cudaSuccess)
        return fail(c, UPIC_ERR_CUDA, "cudaFuncSetAttribute (implicit map) failed");
    const int occ = implicit_map_occupancy(s->tg, s->order, split, s->picard);
    s->grid = c->nsm * (occ > 0 ? occ : 1);
    // Gauss rules.  With knot splitting, every orbit integrand within a
    // segment -- S_a S_b, (1-s) S'_a S_b, s S'_a S_b in 2D, S_a, (1-s) S'_a,
    // s S'_a on a grid one cell high, the time-interpolated A included -- is
    // a polynomial of degree <= 2 order + 1 in s, which an (order+1)-point
    // Gauss rule integrates exactly, as the deck's nq-point rule does when
    // nq >= order+1: the two then differ by rounding only.  So with knot
    // splitting and nq > order+1 both the point-by-point orbit integrals and
    // the segment moments use the (order+1)-point rule; without knot
    // splitting a segment spans several spline pieces and the deck's rule is
    // kept.
    std::vector<double> qs, qw, ms, mw;
    if (split && s->nq > s->order + 1) s->nq = s->order + 1;
    gauss_legendre_01(s->nq, qs, qw);
    s->mnq = s->nq;
    gauss_legendre_01(s->mnq, ms, mw);
    std::vector<double> tab(4 * kMaxQuad, 0.0);
    for (int i = 0; i < s->nq; ++i) {
        tab[i] = qs[i];
        tab[kMaxQuad + i] = qw[i];
    }
    for (int i = 0; i < s->mnq; ++i) {
        tab[2 * kMaxQuad + i] = ms[i];
        tab[3 * kMaxQuad + i] = mw[i];
    }
    int rc;
    if ((rc = dalloc(c, &s->qtab, tab.size()))) return rc;
    if (cudaMemcpy(s->qtab, tab.data(), sizeof(double) * tab.size(), cudaMemcpyHostToDevice) != cudaSuccess)
        return fail(c, UPIC_ERR_CUDA, "quadrature upload failed");
    if ((rc = dalloc(c, &s->spec, 9 * (size_t)N)) || (rc = dalloc(c, &s->spec_out, 9 * (size_t)N)) ||
        (rc = dalloc(c, &s->Jhat, 3 * (size_t)N)) || (rc = dalloc(c, &s->gspec, 5 * (size_t)N)) ||
        (rc = dalloc(c, &s->dspec, 10 * (size_t)N)) || (rc = dalloc(c, &s->dreal, 10 * (size_t)N)) ||
        (rc = dalloc(c, &s->rec, (size_t)kIRec * N)) || (rc = dalloc(c, &s->excl, (size_t)N)) ||
        (rc = dalloc(c, &s->acc, 8 * (size_t)N)) || (rc = dalloc(c, &s->J, 3 * (size_t)N)) ||
        (rc = dalloc(c, &s->Jf, 3 * (size_t)N)) || (rc = dalloc(c, &s->guess, 3 * (size_t)N)) ||
        (rc = dalloc(c, &s->map, 3 * (size_t)N)) || (rc = dalloc(c, &s->trial, 3 * (size_t)N)) ||
        (rc = dalloc(c, &s->trial_map, 3 * (size_t)N)) || (rc = dalloc(c, &s->cand, 3 * (size_t)N)) ||
        (rc = dalloc(c, &s->resid, 3 * (size_t)N)) || (rc = dalloc(c, &s->partials, 64 * (size_t)kNormGrid)) ||
        (rc = dalloc(c, &s->dnorm, 1)) || (rc = dalloc(c, &s->dstats, 1)) || (rc = dalloc(c, &s->ddots, 32)) ||
        (rc = dalloc(c, &s->dflag, 1)) || (rc = dalloc(c, &s->pstat, 4)) || (rc = dalloc(c, &s->perr, 1)))
        return rc;
    if (s->picard && (rc = dalloc(c, &s->Jprev, 3 * (size_t)N))) return rc;
    if (c->cfg.current_predictor == UPIC_PREDICTOR_EXTRAPOLATED && (rc = dalloc(c, &s->Jold, 3 * (size_t)N)))
        return rc;
    if ((rc = dalloc(c, &s->J0, 3 * (size_t)N)) || (rc = dalloc(c, &s->dnorm3, 3))) return rc;
    if (c->cfg.current_predictor != UPIC_PREDICTOR_PREVIOUS && (rc = dalloc(c, &s->Jx, 3 * (size_t)N))) return rc;
    if (c->cfg.current_predictor == UPIC_PREDICTOR_LEARNED) {
        if ((rc = dalloc(c, &s->Jl, 3 * (size_t)N)) || (rc = dalloc(c, &s->fbuf, 4 * (size_t)N)) ||
            (rc = dalloc(c, &s->dloss, 1)))
            return rc;
        const cudaError_t e = gnet::net_create(&s->net, c->nx, c->ny, c->cfg.learned_seed, c->nsm);
        if (e != cudaSuccess)
            return fail(c, UPIC_ERR_NOMEM, std::string("learned predictor: ") + cudaGetErrorString(e));
    }
    for (int k = 0; k < kHist; ++k)
        if ((rc = dalloc(c, &s->hx[k], 3 * (size_t)N)) || (rc = dalloc(c, &s->hr[k], 3 * (size_t)N))) return rc;
    if (cudaMallocHost(&s->hnorm, sizeof(NormSums)) != cudaSuccess ||
        cudaMallocHost(&s->hstats, sizeof(MapStats)) != cudaSuccess ||
        cudaMallocHost(&s->hdots, sizeof(double) * 32) != cudaSuccess ||
        cudaMallocHost(&s->hflag, sizeof(int)) != cudaSuccess ||
        cudaMallocHost(&s->hnorm3, sizeof(NormSums) * 3) != cudaSuccess ||
        cudaMallocHost(&s->hloss, sizeof(double)) != cudaSuccess ||
        cudaMallocHost(&s->hcon, sizeof(double) * 4 * (size_t)std::max(1, c->cfg.nonlinear_max_iter)) != cudaSuccess)
        return fail(c, UPIC_ERR_NOMEM, "cudaMallocHost failed");
    if ((rc = dalloc(c, &s->dcon, 4 * (size_t)std::max(1, c->cfg.nonlinear_max_iter)))) return rc;
    std::vector<unsigned char> ex(N, 0);
    for (int i = 0; i < c->nx; ++i)
        for (int j = 0; j < c->ny; ++j)
            ex[i * c->ny + j] = (is_even_nyquist(i, c->nx) || is_even_nyquist(j, c->ny)) ? 1 : 0;
    if (cudaMemcpy(s->excl, ex.data(), N, cudaMemcpyHostToDevice) != cudaSuccess)
        return fail(c, UPIC_ERR_CUDA, "mask upload failed");
    return 0;
}

void implicit_destroy(upic_ctx* c) {
    if (!c || !c->imp) return;
    ImplicitState* s = c->imp;
    if (s->hnorm) cudaFreeHost(s->hnorm);
    if (s->hstats) cudaFreeHost(s->hstats);
    if (s->hdots) cudaFreeHost(s->hdots);
    if (s->hflag) cudaFreeHost(s->hflag);
    if (s->hnorm3) cudaFreeHost(s->hnorm3);
    if (s->hloss) cudaFreeHost(s->hloss);
    if (s->hcon) cudaFreeHost(s->hcon);
    gnet::net_destroy(s->net);
    delete s;
    c->imp = nullptr;
}

int implicit_set_particles(upic_ctx* c, long np, const double* x, const double* y, const double* P,
                           const double* v, const double* v_prev, const double* q, const double* m) {
    ImplicitState& s = *c->imp;
    const HostScan hs = scan_particles(np, x, y, v, q, m);
    if (!hs.finite) return fail(c, UPIC_ERR_NONFINITE, "non-finite particle position or velocity");
    // gamma_from_v (:623)
    if (!s.picard && hs.speed_max >= c->cfg.kappa)
        return fail(c, UPIC_ERR_SUPERLUMINAL, "relativistic initial velocity must satisfy |v| < kappa");
    if (!hs.positive_m) return fail(c, UPIC_ERR_ARGUMENT, "particle masses must be positive");
    const bool uniform = hs.uniform;
    const double qabs = hs.qabs;
    int rc;
    if (np > s.cap || (!uniform && !s.P[0].q)) {
        free_particles(c, s);
        if ((rc = alloc_particles(c, s, std::max(np, s.cap), !uniform))) return rc;
    }
    if ((rc = ensure_tmp3(c, np))) return rc;
    s.np = np;
    s.tg.chunk = choose_chunk(np, s.grid, kMaxImplicitChunk);
    s.cur = 0;
    s.uniform = uniform;
    s.q0 = np ? q[0] : 0.0;
    s.m0 = np ? m[0] : 0.0;
    s.qabs = qabs;
    ParticleSoA& d = s.P[0];
    if (np > 0) {
        UPIC_CUDA(c, cudaMemcpyAsync(d.x, x, sizeof(double) * np, cudaMemcpyHostToDevice, c->st));
        UPIC_CUDA(c, cudaMemcpyAsync(d.y, y, sizeof(double) * np, cudaMemcpyHostToDevice, c->st));
        wrap_positions_kernel<<<gridn(np), 256, 0, c->st>>>(d.x, d.y, np, c->cfg.Lx, c->cfg.Ly);
        count_launches(1);
        if ((rc = upload3(c, P, np, d.Px, d.Py, d.Pz))) return rc;
        if ((rc = upload3(c, v, np, d.vx, d.vy, d.vz))) return rc;
        if ((rc = upload3(c, v_prev, np, d.wx, d.wy, d.wz))) return rc;
        UPIC_CUDA(c, cudaMemcpyAsync(s.bx[0], d.vx, sizeof(double) * np, cudaMemcpyDeviceToDevice, c->st));
        UPIC_CUDA(c, cudaMemcpyAsync(s.by[0], d.vy, sizeof(double) * np, cudaMemcpyDeviceToDevice, c->st));
        UPIC_CUDA(c, cudaMemcpyAsync(s.bz[0], d.vz, sizeof(double) * np, cudaMemcpyDeviceToDevice, c->st));
        if (!uniform) {
            UPIC_CUDA(c, cudaMemcpyAsync(d.q, q, sizeof(double) * np, cudaMemcpyHostToDevice, c->st));
            UPIC_CUDA(c, cudaMemcpyAsync(d.m, m, sizeof(double) * np, cudaMemcpyHostToDevice, c->st));
        }
        if ((rc = iota(c, d.id, np))) return rc;
    }
    // fixed-point bound of the orbit-averaged current: |v| < kappa; for the
    // non-relativistic method 16 times the larger of the initial speeds and c
    double bJ = qabs * c->cfg.kappa / s.dV;
    if (s.picard) {
        const double vmax = std::max(c->cfg.c, hs.comp_max);
        bJ = qabs * 16.0 * vmax / s.dV;
        s.vb_limit = 16.0 * vmax;
    }
    s.scaleJ[0] = s.scaleJ[1] = s.scaleJ[2] = fixed_scale(bJ);
    s.scaleJ[3] = fixed_scale(qabs / s.dV);
    s.ready = false;
    s.energy_valid = false;
    s.loaded = true;
    s.steps = 0;
    return sync(c);
}

void implicit_mark_unloaded(upic_ctx* c) {
    ImplicitState& s = *c->imp;
    s.np = 0;
    s.loaded = false;
    s.ready = false;
    s.energy_valid = false;
}

// Everything the next implicit step reads: the particle set with its orbit
// velocities, the state spectra, the state current (the next step's first
// current guess), scales and counters.
int implicit_state_io(upic_ctx* c, StateIO& io) {
    ImplicitState& s = *c->imp;
    int rc;
    long np = s.np;
    int uniform = s.uniform ? 1 : 0, loaded = s.loaded ? 1 : 0, ready = s.ready ? 1 : 0,
        evalid = s.energy_valid ? 1 : 0;
    if ((rc = state_value(c, io, np)) || (rc = state_value(c, io, uniform)) || (rc = state_value(c, io, loaded)) ||
        (rc = state_value(c, io, ready)) || (rc = state_value(c, io, evalid)) ||
        (rc = state_value(c, io, s.energy_W)) || (rc = state_value(c, io, s.energy_K)) ||
        (rc = state_value(c, io, s.q0)) || (rc = state_value(c, io, s.m0)) || (rc = state_value(c, io, s.qabs)) ||
        (rc = state_value(c, io, s.vb_limit)) || (rc = state_bytes(c, io, s.scaleJ, sizeof(s.scaleJ))) ||
        (rc = state_value(c, io, s.steps)))
        return rc;
    if (!io.writing) {
        if (np < 0 || np > 0x7fffffffL) return fail(c, UPIC_ERR_ARGUMENT, "state file: bad particle count");
        if (np > s.cap || (!uniform && !s.P[0].q)) {
            free_particles(c, s);
            if ((rc = alloc_particles(c, s, std::max(np, s.cap), !uniform))) return rc;
        }
        if ((rc = ensure_tmp3(c, np))) return rc;
        s.cur = 0;
        s.np = np;
        s.tg.chunk = choose_chunk(np, s.grid, kMaxImplicitChunk);
        s.uniform = uniform != 0;
        s.loaded = loaded != 0;
        s.ready = ready != 0;
        s.energy_valid = evalid != 0;
        c->np = np;
        c->fields_ready = s.ready;
        c->steps = s.steps;
    }
    ParticleSoA& p = s.P[s.cur];
    const size_t pb = sizeof(double) * np;
    double* arrs[] = {p.x, p.y, p.Px, p.Py, p.Pz, p.vx, p.vy, p.vz, p.wx, p.wy, p.wz,
                      s.bx[s.cur], s.by[s.cur], s.bz[s.cur]};
    for (double* a : arrs)
        if ((rc = state_device(c, io, a, pb))) return rc;
    if ((rc = state_device(c, io, p.id, sizeof(int) * np))) return rc;
    if (!uniform && ((rc = state_device(c, io, p.q, pb)) || (rc = state_device(c, io, p.m, pb)))) return rc;
    const size_t N = (size_t)c->N;
    if ((rc = state_device(c, io, s.spec, sizeof(double2) * 9 * N)) ||
        (rc = state_device(c, io, s.J, sizeof(double) * 3 * N)))
        return rc;
    if (s.Jold) {
        int have = s.have_Jold ? 1 : 0;
        if ((rc = state_value(c, io, have)) || (rc = state_device(c, io, s.Jold, sizeof(double) * 3 * N))) return rc;
        s.have_Jold = have != 0;
    }
    if (s.net) {
        int newest = 0, count = 0, use = s.use_learned ? 1 : 0;
        long t = 0;
        gnet::net_host_state(s.net, &newest, &count, &t, false);
        if ((rc = state_value(c, io, newest)) || (rc = state_value(c, io, count)) || (rc = state_value(c, io, t)) ||
            (rc = state_value(c, io, use)) || (rc = state_value(c, io, s.trained_steps)))
            return rc;
        if (!io.writing) {
            if (newest < -1 || newest >= gnet::kFrames || count < 0 || count > gnet::kFrames || t < 0)
                return fail(c, UPIC_ERR_ARGUMENT, "state file: bad learned-predictor state");
            gnet::net_host_state(s.net, &newest, &count, &t, true);
            s.use_learned = use != 0;
        }
        void* ptrs[16];
        size_t sizes[16];
        const size_t k = gnet::net_state_ranges(s.net, ptrs, sizes, 16);
        for (size_t i = 0; i < k; ++i)
            if ((rc = state_device(c, io, ptrs[i], sizes[i]))) return rc;
    }
    return 0;
}

int implicit_get_particles(upic_ctx* c, long np, double* x, double* y, double* P, double* v, double* v_prev) {
    ImplicitState& s = *c->imp;
    if (np != s.np) return fail(c, UPIC_ERR_ARGUMENT, "particle count does not match the context");
    if (np == 0) return UPIC_OK;
    ParticleSoA src = s.P[s.cur];
    ParticleSoA dst = s.P[1 - s.cur];
    UPIC_CUDA(c, unpermute_particles(src, dst, np, c->st));
    int rc;
    if (x) UPIC_CUDA(c, cudaMemcpyAsync(x, dst.x, sizeof(double) * np, cudaMemcpyDeviceToHost, c->st));
    if (y) UPIC_CUDA(c, cudaMemcpyAsync(y, dst.y, sizeof(double) * np, cudaMemcpyDeviceToHost, c->st));
    if (P && (rc = download3(c, P, np, dst.Px, dst.Py, dst.Pz))) return rc;
    if ((rc = sync(c))) return rc;
    if (v && (rc = download3(c, v, np, dst.vx, dst.vy, dst.vz))) return rc;
    if ((rc = sync(c))) return rc;
    if (v_prev && (rc = download3(c, v_prev, np, dst.wx, dst.wy, dst.wz))) return rc;
    return sync(c);
}

int implicit_init_fields(upic_ctx* c, double* diag_row) {
    ImplicitState& s = *c->imp;
    const upic_config& cf = c->cfg;
    const int N = c->N;
    if (!s.loaded) return fail(c, UPIC_ERR_STATE, "upic_set_particles first");
    int rc;
    if (s.np > 0 && (rc = sort_active(c, s))) return rc;
    ParticleSoA& p = s.P[s.cur];
    // rho_e, J by point deposit (deposit_scalar_to_mesh :2117, deposit_current_to_mesh :2182)
    UPIC_CUDA(c, cudaMemsetAsync(s.acc, 0, sizeof(unsigned long long) * 8 * (size_t)N, c->st));
    if (s.np > 0) {
        PointDepositArgs d{};
        d.x = p.x; d.y = p.y; d.vx = p.vx; d.vy = p.vy; d.vz = p.vz;
        d.q = s.uniform ? nullptr : p.q;
        d.q0 = s.q0;
        d.np = s.np;
        d.nx = c->nx; d.ny = c->ny;
        d.Lx = cf.Lx; d.Ly = cf.Ly; d.inv_dx = 1.0 / s.dx; d.inv_dy = 1.0 / s.dy; d.inv_dV = 1.0 / s.dV;
        d.acc = s.acc;
        for (int k = 0; k < 4; ++k) d.scale[k] = s.scaleJ[k];
        UPIC_CUDA(c, launch_point_deposit(s.order, d, c->st));
    }
    // rho = rho_e + n0 with its mean subtracted and the Nyquist planes
    // projected out (project_initial_state :3399) is, in k-space, the
    // spectrum of rho_e with the k = 0 and excluded modes zeroed: the
    // uniform background only enters the k = 0 mode.
    double* rho = s.dreal;
    UPIC_CUDA(c, launch_convert_acc(s.acc, N, s.scaleJ, s.J, rho, 0.0, 3, c->st));
    if (cf.nyquist_projection) UPIC_CUDA(c, launch_project_nyquist(s.J, 3, c->nx, c->ny, c->st));
    // spectra: phi from Poisson (solve_periodic_poisson_for_phi :3196), psi = A = U = 0
    UPIC_CUDA(c, cudaMemsetAsync(s.spec, 0, sizeof(double2) * 9 * (size_t)N, c->st));
    UPIC_CUDA(c, fft2d_batched(c->plan, s.spec + 2 * (size_t)N, 1, 0, c->st, rho));
    UPIC_CUDA(c, launch_kspace_mask(s.spec + 2 * (size_t)N, 1, N, cf.nyquist_projection ? s.excl : nullptr, 1,
                                    c->st));
    UPIC_CUDA(c, launch_poisson_kspace(N, c->d_k2, s.spec + 2 * (size_t)N, s.picard ? cf.eps0 : 1.0 / cf.sigma1,
                                       s.spec, c->st));
    UPIC_CUDA(c, launch_kspace_mask(s.spec, 1, N, cf.nyquist_projection ? s.excl : nullptr, 1, c->st));
    const bool with_AU = s.init_AU_set && !s.picard;
    if (with_AU) {
        // A, U of upic_set_initial_potential, Nyquist-projected with the rest
        // of the start state (project_initial_state :3398)
        UPIC_CUDA(c, fft2d_batched(c->plan, s.spec + 3 * (size_t)N, 3, 0, c->st, s.init_AU));
        UPIC_CUDA(c, fft2d_batched(c->plan, s.spec + 6 * (size_t)N, 3, 0, c->st, s.init_AU + 3 * (size_t)N));
        if (cf.nyquist_projection) UPIC_CUDA(c, launch_kspace_mask(s.spec + 3 * (size_t)N, 6, N, s.excl, 0, c->st));
        s.init_AU_set = false;
    }
    // P = m gamma v + q A (A = 0 unless set); v_prev from one backward Lorentz step; vbar = v
    if (s.np > 0 && s.picard) {
        // P = m v, v_prev = v - dt (q/m) E (ec_pic_serial_demo.cpp:1200-1210)
        UPIC_CUDA(c, launch_diag_spectra(N, c->d_kx, c->d_ky, s.spec, s.dspec, c->st));
        UPIC_CUDA(c, fft2d_batched(c->plan, s.dspec, 3, 1, c->st, nullptr, 1, s.dreal));
        UPIC_CUDA(c, launch_picard_startup(s.order, c->nx, c->ny, cf.Lx, cf.Ly, s.dreal, s.np, p.x, p.y, p.vx, p.vy,
                                           p.vz, s.uniform ? nullptr : p.q, s.q0, s.uniform ? nullptr : p.m, s.m0,
                                           cf.dt, p.Px, p.Py, p.Pz, p.wx, p.wy, p.wz, c->st));
    } else if (s.np > 0) {
        UPIC_CUDA(c, launch_momentum_from_v(s.np, p.vx, p.vy, p.vz, s.uniform ? nullptr : p.m, s.m0, cf.kappa,
                                            p.Px, p.Py, p.Pz, c->st));
        if (with_AU) {
            // the projected A in real space, gathered at the particles
            UPIC_CUDA(c, cudaMemcpyAsync(s.dspec, s.spec + 3 * (size_t)N, sizeof(double2) * 3 * N,
                                         cudaMemcpyDeviceToDevice, c->st));
            UPIC_CUDA(c, fft2d_batched(c->plan, s.dspec, 3, 1, c->st, nullptr, 1, s.dreal));
            UPIC_CUDA(c, launch_add_qA(s.order, c->nx, c->ny, cf.Lx, cf.Ly, s.dreal, s.np, p.x, p.y,
                                       s.uniform ? nullptr : p.q, s.q0, p.Px, p.Py, p.Pz, c->st));
        }
        UPIC_CUDA(c, launch_diag_spectra(N, c->d_kx, c->d_ky, s.spec, s.dspec, c->st));
        UPIC_CUDA(c, fft2d_batched(c->plan, s.dspec, 6, 1, c->st, nullptr, 1, s.dreal));
        UPIC_CUDA(c, launch_history_velocity(s.order, c->nx, c->ny, cf.Lx, cf.Ly, s.dreal, s.dreal + 3 * (size_t)N,
                                             s.np, p.x, p.y, p.vx, p.vy, p.vz, s.uniform ? nullptr : p.q, s.q0,
                                             s.uniform ? nullptr : p.m, s.m0, cf.kappa, cf.dt, p.wx, p.wy, p.wz,
                                             c->st));
        const size_t pb = sizeof(double) * s.np;
        UPIC_CUDA(c, cudaMemcpyAsync(s.bx[s.cur], p.vx, pb, cudaMemcpyDeviceToDevice, c->st));
        UPIC_CUDA(c, cudaMemcpyAsync(s.by[s.cur], p.vy, pb, cudaMemcpyDeviceToDevice, c->st));
        UPIC_CUDA(c, cudaMemcpyAsync(s.bz[s.cur], p.vz, pb, cudaMemcpyDeviceToDevice, c->st));
    }
    s.ready = true;
    s.steps = 0;
    s.have_Jold = false;
    c->steps = 0;
    c->fields_ready = true;
    if (s.net) {
        // the learned predictor's frames restart from this state; its
        // weights keep what they learned
        int newest = -1, count = 0;
        long t = 0;
        gnet::net_host_state(s.net, &newest, &count, &t, false);
        newest = -1;
        count = 0;
        gnet::net_host_state(s.net, &newest, &count, &t, true);
        s.use_learned = false;
        if ((rc = push_frame(c, s))) return rc;
    }
    if ((rc = sync(c))) return rc;
    s.energy_valid = false;
    if (diag_row) {
        if ((rc = state_diagnostics(c, s, diag_row))) return rc;
        s.energy_W = diag_row[UPIC_P3_FIELD_ENERGY];
        s.energy_K = diag_row[UPIC_P3_KINETIC_ENERGY];
        s.energy_valid = true;
    }
    return UPIC_OK;
}

int implicit_get_field(upic_ctx* c, int which, double* host) {
    ImplicitState& s = *c->imp;
    const int N = c->N;
    if (which >= UPIC_FIELD_JX && which <= UPIC_FIELD_JZ) {
        UPIC_CUDA(c, cudaMemcpyAsync(host, s.J + (size_t)(which - UPIC_FIELD_JX) * N, sizeof(double) * N,
                                     cudaMemcpyDeviceToHost, c->st));
        return sync(c);
    }
    if (which >= UPIC_FIELD_EX && which <= UPIC_FIELD_BZ) {
        // E = -grad phi - U, B = curl A of the accepted state (compute_E
        // :3338, spectral_curl :1780): diag_spectra slots E 0..2, B 3..5
        UPIC_CUDA(c, launch_diag_spectra(N, c->d_kx, c->d_ky, s.spec, s.dspec, c->st));
        const int slot = which - UPIC_FIELD_EX;
        UPIC_CUDA(c, fft2d_batched(c->plan, s.dspec + (size_t)slot * N, 1, 1, c->st, nullptr, 1, s.dreal));
        UPIC_CUDA(c, cudaMemcpyAsync(host, s.dreal, sizeof(double) * N, cudaMemcpyDeviceToHost, c->st));
        return sync(c);
    }
    // spectra slot of each field: phi 0, psi 1, rho 2, A 3..5, U 6..8
    int slot;
    switch (which) {
        case UPIC_FIELD_PHI: slot = 0; break;
        case UPIC_FIELD_PSI: slot = 1; break;
        case UPIC_FIELD_RHO: slot = 2; break;
        case UPIC_FIELD_AX: case UPIC_FIELD_AY: case UPIC_FIELD_AZ: slot = 3 + which - UPIC_FIELD_AX; break;
        case UPIC_FIELD_UX: case UPIC_FIELD_UY: case UPIC_FIELD_UZ: slot = 6 + which - UPIC_FIELD_UX; break;
        default: return fail(c, UPIC_ERR_ARGUMENT, "unknown field");
    }
    UPIC_CUDA(c, cudaMemcpyAsync(s.dspec, s.spec + (size_t)slot * N, sizeof(double2) * N, cudaMemcpyDeviceToDevice,
                                 c->st));
    UPIC_CUDA(c, fft2d_batched(c->plan, s.dspec, 1, 1, c->st, nullptr, 1, s.dreal));
    UPIC_CUDA(c, cudaMemcpyAsync(host, s.dreal, sizeof(double) * N, cudaMemcpyDeviceToHost, c->st));
    return sync(c);
}

// compute_step_diagnostics (:4501 -> :4340) of the step just accepted: the
// state before it is the spare particle set and spec_out, the state after it
// the current set and spec.  W0, K0, W1, K1: field and kinetic energies.
int step_diagnostics(upic_ctx* c, ImplicitState& s, double W0, double K0, double W1, double K1, double* out) {
    const upic_config& cf = c->cfg;
    const int N = c->N;
    int rc;
    if (!s.sd_spec) {
        if ((rc = dalloc(c, &s.sd_spec, 12 * (size_t)N)) || (rc = dalloc(c, &s.sd_rec, 12 * (size_t)N)) ||
            (rc = dalloc(c, &s.sd_counts, 4)))
            return rc;
    }
    const double* Jgrid = s.J;
    if (s.picard && s.np > 0) {
        // Project1 (compute_step_diagnostics, ec_pic_serial_demo.cpp:1384):
        // vbar = (v^{n+1} + v^n) / 2 and the grid work of its re-deposited
        // orbit current
        const ParticleSoA& v1 = s.P[s.cur];
        const ParticleSoA& v0 = s.P[1 - s.cur];
        UPIC_CUDA(c, launch_half_sum((int)s.np, v1.vx, v0.vx, s.bx[s.cur], c->st));
        UPIC_CUDA(c, launch_half_sum((int)s.np, v1.vy, v0.vy, s.by[s.cur], c->st));
        UPIC_CUDA(c, launch_half_sum((int)s.np, v1.vz, v0.vz, s.bz[s.cur], c->st));
        UPIC_CUDA(c, cudaMemsetAsync(s.acc, 0, sizeof(unsigned long long) * 6 * (size_t)N, c->st));
        UPIC_CUDA(c, cudaMemsetAsync(s.dstats, 0, sizeof(MapStats), c->st));
        ImplicitMapArgs a{};
        a.x = v0.x; a.y = v0.y; a.vx = v0.vx; a.vy = v0.vy; a.vz = v0.vz;
        a.q = v0.q; a.q0 = s.q0; a.id = v0.id;
        a.gx = v1.vx; a.gy = v1.vy; a.gz = v1.vz;
        a.vb_limit = INFINITY;
        a.np = s.np;
        a.Lx = cf.Lx; a.Ly = cf.Ly; a.inv_dx = 1.0 / s.dx; a.inv_dy = 1.0 / s.dy; a.inv_dV = 1.0 / s.dV;
        a.dt = cf.dt; a.kappa = cf.kappa;
        a.split = cf.split_orbit_at_knots;
        a.chunks = s.sw.chunks;
        a.nchunks = s.sw.nchunks;
        a.acc = s.acc;
        for (int d = 0; d < 3; ++d) a.scale[d] = s.scaleJ[d];
        a.stats = s.dstats;
        a.qtab = s.qtab;
        a.nq = s.nq;
        a.mnq = s.mnq;
        UPIC_CUDA(c, launch_implicit_map(s.order, s.uniform, a.split != 0, s.tg, a, s.grid, c->st, true));
        UPIC_CUDA(c, launch_convert_acc(s.acc, N, s.scaleJ, s.trial, nullptr, 0.0, 1, c->st));
        Jgrid = s.trial;
    }
    UPIC_CUDA(c, launch_step_diag_spectra(N, c->d_kx, c->d_ky, s.spec_out, s.spec, s.sd_spec, c->st));
    UPIC_CUDA(c, fft2d_batched(c->plan, s.sd_spec, 12, 1, c->st, nullptr, 2, s.sd_rec, 12, 0));
    UPIC_CUDA(c, cudaMemsetAsync(s.sd_counts, 0, sizeof(unsigned long long) * 4, c->st));
    const ParticleSoA& p0 = s.P[1 - s.cur];
    StepDiagArgs a{};
    a.x = p0.x;
    a.y = p0.y;
    a.bx = s.bx[s.cur];
    a.by = s.by[s.cur];
    a.bz = s.bz[s.cur];
    a.q = s.uniform ? nullptr : s.P[s.cur].q;
    a.q0 = s.q0;
    a.np = s.np;
    a.nx = c->nx;
    a.ny = c->ny;
    a.Lx = cf.Lx;
    a.Ly = cf.Ly;
    a.inv_dx = 1.0 / s.dx;
    a.inv_dy = 1.0 / s.dy;
    a.dt = cf.dt;
    a.split = cf.split_orbit_at_knots;
    a.nq = s.nq;
    a.qtab = s.qtab;
    a.rec = s.sd_rec;
    a.partials = s.partials;
    a.counts = s.sd_counts;
    if (!s.picard && s.last_refined > 0) {
        // sub-cycled particles (compute_subcycled_step_diagnostics :4363):
        // one A-chain term per recorded sub-orbit
        a.nsub = s.nsub;
        a.refined = s.refined;
        a.nref = s.last_refined;
        a.roff = s.roff;
        a.sub = s.sub_rec;
        // partials hold 64 x kNormGrid doubles: the main kernel's 16 x kNormGrid,
        // then up to 16 x 2 kNormGrid for the refined blocks
        a.refined_grid_max = 2 * kNormGrid;
    }
    UPIC_CUDA(c, launch_step_diag(s.order, a, kNormGrid, s.ddots, c->st));
    UPIC_CUDA(c, launch_grid_work(N, Jgrid, s.sd_rec, s.partials + 16 * kNormGrid, kNormGrid, s.ddots + 14, c->st));
    unsigned long long cnt[4];
    UPIC_CUDA(c, cudaMemcpyAsync(s.hdots, s.ddots, sizeof(double) * 16, cudaMemcpyDeviceToHost, c->st));
    UPIC_CUDA(c, cudaMemcpyAsync(cnt, s.sd_counts, sizeof(cnt), cudaMemcpyDeviceToHost, c->st));
    if ((rc = sync(c))) return rc;
    const double* h = s.hdots;
    auto tot = [&](int k) { return h[2 * k] + h[2 * k + 1]; };
    const double denom = (double)std::max<long>(1, 3 * s.np);
    const double arms = std::sqrt(tot(1) / denom), rhsrms = std::sqrt(tot(2) / denom);
    double* o = out;
    o[UPIC_SD_A_CHAIN_ABS_RMS] = std::sqrt(tot(0) / denom);
    o[UPIC_SD_A_CHAIN_REL_RMS] = o[UPIC_SD_A_CHAIN_ABS_RMS] / (0.5 * (arms + rhsrms) + 1.0e-300);
    o[UPIC_SD_A_CHAIN_MAX_NORM] = h[12];
    o[UPIC_SD_A_CHAIN_MEAN_NORM] = tot(3) / (double)std::max<long>(1, s.np);
    o[UPIC_SD_A_CHAIN_WORK_DEFECT] = tot(4);
    o[UPIC_SD_DELTA_K] = K1 - K0;
    o[UPIC_SD_DELTA_W] = W1 - W0;
    o[UPIC_SD_DELTA_TOTAL_ENERGY] = o[UPIC_SD_DELTA_K] + o[UPIC_SD_DELTA_W];
    o[UPIC_SD_PARTICLE_WORK] = tot(5);
    o[UPIC_SD_GRID_WORK] = cf.dt * (h[14] + h[15]) * s.dV;
    o[UPIC_SD_DEPOSIT_GATHER_WORK_RESIDUAL] = o[UPIC_SD_PARTICLE_WORK] - o[UPIC_SD_GRID_WORK];
    o[UPIC_SD_PARTICLE_ENERGY_RESIDUAL] = o[UPIC_SD_DELTA_K] - o[UPIC_SD_PARTICLE_WORK];
    o[UPIC_SD_FIELD_ENERGY_RESIDUAL] = o[UPIC_SD_DELTA_W] + o[UPIC_SD_GRID_WORK];
    o[UPIC_SD_CROSSING_PARTICLES] = (double)cnt[2];
    o[UPIC_SD_TOTAL_CROSSINGS] = (double)cnt[1];
    o[UPIC_SD_AVERAGE_PATH_SEGMENTS] = s.np ? (double)cnt[0] / (double)s.np : 1.0;
    o[UPIC_SD_MAX_PATH_SEGMENTS] = (double)(s.np ? cnt[3] : 1);
    return 0;
}

int orbit_stage(upic_ctx* c, ImplicitState& s, long np) {
    int rc;
    if (!s.ogrid) {
        if ((rc = dalloc(c, &s.ogrid, 9 * (size_t)c->N)) || (rc = dalloc(c, &s.oerr, 1))) return rc;
    }
    if (np <= s.ocap) return 0;
    double** bufs[] = {&s.ox, &s.oy, &s.odx, &s.ovb, &s.oq, &s.ogat, &s.ograd};
    const long sizes[] = {1, 1, 3, 3, 1, 3, 9};
    for (int k = 0; k < 7; ++k) {
        dfree(c, *bufs[k]);
        *bufs[k] = nullptr;
        if ((rc = dalloc(c, bufs[k], sizes[k] * (size_t)np))) return rc;
    }
    s.ocap = np;
    return 0;
}

OrbitArgs orbit_args(upic_ctx* c, ImplicitState& s, long np) {
    const upic_config& cf = c->cfg;
    OrbitArgs a{};
    a.x = s.ox; a.y = s.oy; a.dx = s.odx; a.vbar = s.ovb; a.q = s.oq;
    a.np = np;
    a.nx = c->nx; a.ny = c->ny;
    a.Lx = cf.Lx; a.Ly = cf.Ly; a.inv_dx = 1.0 / s.dx; a.inv_dy = 1.0 / s.dy; a.inv_dV = 1.0 / s.dV;
    a.split = cf.split_orbit_at_knots;
    a.nq = s.nq;
    a.qtab = s.qtab;
    a.acc = s.acc;
    a.err = s.oerr;
    return a;
}

int orbit_check(upic_ctx* c, ImplicitState& s) {
    UPIC_CUDA(c, cudaMemcpyAsync(s.hflag, s.oerr, sizeof(int), cudaMemcpyDeviceToHost, c->st));
    const int rc = sync(c);
    if (rc) return rc;
    if (*s.hflag)
        return fail(c, UPIC_ERR_TOO_LARGE, "an orbit crosses more spline knots than the kernel holds (38)");
    return 0;
}

}  // namespace upic_host

using namespace upic_host;

extern "C" int upic_orbit_deposit(upic_ctx* c, long np, const double* x, const double* y, const double* dx,
                                  const double* vbar, const double* q, double* J) {
    if (!c) return UPIC_ERR_ARGUMENT;
    if (!c->imp) return fail(c, UPIC_ERR_STATE, "context was not created with UPIC_METHOD_CN_ORBIT");
    if (!J || np < 0 || (np > 0 && (!x || !y || !dx || !vbar || !q)))
        return fail(c, UPIC_ERR_ARGUMENT, "null array or negative particle count");
    ImplicitState& s = *c->imp;
    const int N = c->N;
    int rc;
    if ((rc = orbit_stage(c, s, np))) return rc;
    double qabs = 0.0, vmax = 0.0;
    for (long p = 0; p < np; ++p) {
        qabs += std::fabs(q[p]);
        for (int d = 0; d < 3; ++d) vmax = std::max(vmax, std::fabs(vbar[3 * p + d]));
        if (!std::isfinite(q[p]) || !std::isfinite(x[p]) || !std::isfinite(y[p]))
            return fail(c, UPIC_ERR_NONFINITE, "non-finite particle input");
    }
    if (!std::isfinite(vmax)) return fail(c, UPIC_ERR_NONFINITE, "non-finite orbit velocity");
    OrbitArgs a = orbit_args(c, s, np);
    const double scale = fixed_scale(qabs * vmax / s.dV);
    double sc4[4] = {scale, scale, scale, 1.0};
    for (int k = 0; k < 3; ++k) a.scale[k] = scale;
    UPIC_CUDA(c, cudaMemsetAsync(s.acc, 0, sizeof(unsigned long long) * 6 * (size_t)N, c->st));
    UPIC_CUDA(c, cudaMemsetAsync(s.oerr, 0, sizeof(int), c->st));
    if (np > 0) {
        UPIC_CUDA(c, cudaMemcpyAsync(s.ox, x, sizeof(double) * np, cudaMemcpyHostToDevice, c->st));
        UPIC_CUDA(c, cudaMemcpyAsync(s.oy, y, sizeof(double) * np, cudaMemcpyHostToDevice, c->st));
        UPIC_CUDA(c, cudaMemcpyAsync(s.odx, dx, sizeof(double) * 3 * np, cudaMemcpyHostToDevice, c->st));
        UPIC_CUDA(c, cudaMemcpyAsync(s.ovb, vbar, sizeof(double) * 3 * np, cudaMemcpyHostToDevice, c->st));
        UPIC_CUDA(c, cudaMemcpyAsync(s.oq, q, sizeof(double) * np, cudaMemcpyHostToDevice, c->st));
        UPIC_CUDA(c, launch_orbit_deposit(s.order, a, c->st));
    }
    double* out = s.dreal;
    UPIC_CUDA(c, launch_convert_acc(s.acc, N, sc4, out, nullptr, 0.0, 1, c->st));
    if (c->cfg.nyquist_projection) UPIC_CUDA(c, launch_project_nyquist(out, 3, c->nx, c->ny, c->st));
    UPIC_CUDA(c, cudaMemcpyAsync(J, out, sizeof(double) * 3 * N, cudaMemcpyDeviceToHost, c->st));
    return orbit_check(c, s);
}

extern "C" int upic_orbit_gather(upic_ctx* c, long np, const double* x, const double* y, const double* dx,
                                 const double* mesh, const double* An, const double* Anp1, double* gathered,
                                 double* grad) {
    if (!c) return UPIC_ERR_ARGUMENT;
    if (!c->imp) return fail(c, UPIC_ERR_STATE, "context was not created with UPIC_METHOD_CN_ORBIT");
    if (!mesh || !An || !Anp1 || np < 0 || (np > 0 && (!x || !y || !dx || !gathered || !grad)))
        return fail(c, UPIC_ERR_ARGUMENT, "null array or negative particle count");
    ImplicitState& s = *c->imp;
    const int N = c->N;
    int rc;
    if ((rc = orbit_stage(c, s, np))) return rc;
    OrbitArgs a = orbit_args(c, s, np);
    a.mesh = s.ogrid;
    a.An = s.ogrid + 3 * (size_t)N;
    a.Ae = s.ogrid + 6 * (size_t)N;
    a.gathered = s.ogat;
    a.grad = s.ograd;
    UPIC_CUDA(c, cudaMemsetAsync(s.oerr, 0, sizeof(int), c->st));
    UPIC_CUDA(c, cudaMemcpyAsync(s.ogrid, mesh, sizeof(double) * 3 * N, cudaMemcpyHostToDevice, c->st));
    UPIC_CUDA(c, cudaMemcpyAsync(s.ogrid + 3 * (size_t)N, An, sizeof(double) * 3 * N, cudaMemcpyHostToDevice, c->st));
    UPIC_CUDA(c, cudaMemcpyAsync(s.ogrid + 6 * (size_t)N, Anp1, sizeof(double) * 3 * N, cudaMemcpyHostToDevice,
                                 c->st));
    if (np > 0) {
        UPIC_CUDA(c, cudaMemcpyAsync(s.ox, x, sizeof(double) * np, cudaMemcpyHostToDevice, c->st));
        UPIC_CUDA(c, cudaMemcpyAsync(s.oy, y, sizeof(double) * np, cudaMemcpyHostToDevice, c->st));
        UPIC_CUDA(c, cudaMemcpyAsync(s.odx, dx, sizeof(double) * 3 * np, cudaMemcpyHostToDevice, c->st));
        UPIC_CUDA(c, launch_orbit_gather(s.order, a, c->st));
        UPIC_CUDA(c, cudaMemcpyAsync(gathered, s.ogat, sizeof(double) * 3 * np, cudaMemcpyDeviceToHost, c->st));
        UPIC_CUDA(c, cudaMemcpyAsync(grad, s.ograd, sizeof(double) * 9 * np, cudaMemcpyDeviceToHost, c->st));
    }
    return orbit_check(c, s);
}

namespace {
// Device scratch of one kernel-level call, freed on every return path.
struct Scratch {
    std::vector<void*> p;
    ~Scratch() {
        for (void* q : p) cudaFree(q);
    }
    template <typename T>
    T* get(size_t n) {
        void* v = nullptr;
        if (cudaMalloc(&v, n * sizeof(T) + 16) != cudaSuccess) return nullptr;
        p.push_back(v);
        return reinterpret_cast<T*>(v);
    }
};
}  // namespace

extern "C" int upic_guess_conv(upic_ctx* c, int nx, int ny, const uint16_t* x, const uint16_t* w, const float* bias,
                               const uint16_t* mask, int mode, int sign, void* out) {
    if (!c) return UPIC_ERR_ARGUMENT;
    if (nx < 1 || ny < 1 || (long)nx * ny > (1L << 26) || !x || !w || !out || (sign != 1 && sign != -1) ||
        mode < gnet::kConvRelu || mode > gnet::kConvMask || (mode == gnet::kConvMask && !mask))
        return fail(c, UPIC_ERR_ARGUMENT, "upic_guess_conv: bad grid, mode, sign or null array");
    const size_t P = (size_t)nx * ny, act = P * gnet::kC;
    Scratch sc;
    uint16_t *dx = sc.get<uint16_t>(act), *dw = sc.get<uint16_t>(gnet::kW), *dm = nullptr, *dob = nullptr;
    float *db = nullptr, *dof = nullptr;
    int* derr = sc.get<int>(1);
    if (!dx || !dw || !derr) return fail(c, UPIC_ERR_NOMEM, "upic_guess_conv: device allocation failed");
    if (bias && !(db = sc.get<float>(gnet::kC))) return fail(c, UPIC_ERR_NOMEM, "upic_guess_conv: allocation");
    if (mask && !(dm = sc.get<uint16_t>(act))) return fail(c, UPIC_ERR_NOMEM, "upic_guess_conv: allocation");
    if (mode == gnet::kConvLinear ? !(dof = sc.get<float>(act)) : !(dob = sc.get<uint16_t>(act)))
        return fail(c, UPIC_ERR_NOMEM, "upic_guess_conv: allocation");
    UPIC_CUDA(c, cudaMemcpyAsync(dx, x, sizeof(uint16_t) * act, cudaMemcpyHostToDevice, c->st));
    UPIC_CUDA(c, cudaMemcpyAsync(dw, w, sizeof(uint16_t) * gnet::kW, cudaMemcpyHostToDevice, c->st));
    if (db) UPIC_CUDA(c, cudaMemcpyAsync(db, bias, sizeof(float) * gnet::kC, cudaMemcpyHostToDevice, c->st));
    if (dm) UPIC_CUDA(c, cudaMemcpyAsync(dm, mask, sizeof(uint16_t) * act, cudaMemcpyHostToDevice, c->st));
    UPIC_CUDA(c, cudaMemsetAsync(derr, 0, sizeof(int), c->st));
    gnet::ConvArgs a{};
    a.in = dx;
    a.w = dw;
    a.bias = db;
    a.mask = dm;
    a.out_bf = dob;
    a.out_f = dof;
    a.nx = nx;
    a.ny = ny;
    a.P = (int)P;
    a.sign = sign;
    a.mode = mode;
    a.err = derr;
    UPIC_CUDA(c, mode == gnet::kConvLinear ? gnet::launch_conv_tc_full(a, c->nsm, c->st)
                                           : gnet::launch_conv_tc(a, c->nsm, c->st));
    if (dof) UPIC_CUDA(c, cudaMemcpyAsync(out, dof, sizeof(float) * act, cudaMemcpyDeviceToHost, c->st));
    else UPIC_CUDA(c, cudaMemcpyAsync(out, dob, sizeof(uint16_t) * act, cudaMemcpyDeviceToHost, c->st));
    int herr = 0;
    UPIC_CUDA(c, cudaMemcpyAsync(&herr, derr, sizeof(int), cudaMemcpyDeviceToHost, c->st));
    int rc;
    if ((rc = sync(c))) return rc;
    if (herr) return fail(c, UPIC_ERR_CUDA, "upic_guess_conv: a tensor-core wait timed out");
    return UPIC_OK;
}

extern "C" int upic_guess_wgrad(upic_ctx* c, int nx, int ny, const uint16_t* dz, const uint16_t* x, float* grad) {
    if (!c) return UPIC_ERR_ARGUMENT;
    if (nx < 1 || ny < 1 || (long)nx * ny > (1L << 26) || !dz || !x || !grad)
        return fail(c, UPIC_ERR_ARGUMENT, "upic_guess_wgrad: bad grid or null array");
    const size_t P = (size_t)nx * ny, act = P * gnet::kC;
    const int grid = std::max(1, std::min(2 * c->nsm, (int)((P + 255) / 256)));
    Scratch sc;
    uint16_t *ddz = sc.get<uint16_t>(act), *dx = sc.get<uint16_t>(act);
    float *part = sc.get<float>((size_t)grid * gnet::kParams), *dg = sc.get<float>(gnet::kParams);
    if (!ddz || !dx || !part || !dg) return fail(c, UPIC_ERR_NOMEM, "upic_guess_wgrad: device allocation failed");
    UPIC_CUDA(c, cudaMemcpyAsync(ddz, dz, sizeof(uint16_t) * act, cudaMemcpyHostToDevice, c->st));
    UPIC_CUDA(c, cudaMemcpyAsync(dx, x, sizeof(uint16_t) * act, cudaMemcpyHostToDevice, c->st));
    UPIC_CUDA(c, gnet::launch_conv_wgrad(ddz, dx, nx, ny, part, grid, dg, c->st));
    UPIC_CUDA(c, cudaMemcpyAsync(grad, dg, sizeof(float) * gnet::kParams, cudaMemcpyDeviceToHost, c->st));
    return sync(c);
}

extern "C" int upic_step_implicit(upic_ctx* c, int nsteps, double* diag, double* info, double* step_diag) {
    if (!c) return UPIC_ERR_ARGUMENT;
    if (!c->imp) return fail(c, UPIC_ERR_STATE, "context was not created with UPIC_METHOD_CN_ORBIT");
    ImplicitState& s = *c->imp;
    if (!s.ready) return fail(c, UPIC_ERR_STATE, "upic_init_fields first");
    if (nsteps < 0) return fail(c, UPIC_ERR_ARGUMENT, "nsteps < 0");
    double row[UPIC_P3_DIAG_COUNT];
    s.maplog.clear();
    s.faillog.clear();
    s.fail_event = 0;
    for (int k = 0; k < nsteps; ++k) {
        int rc;
        s.log_step = k;
        if (step_diag && !s.energy_valid) {
            if ((rc = state_diagnostics(c, s, row))) return rc;
            s.energy_W = row[UPIC_P3_FIELD_ENERGY];
            s.energy_K = row[UPIC_P3_KINETIC_ENERGY];
            s.energy_valid = true;
        }
        const double W0 = s.energy_W, K0 = s.energy_K;
        s.energy_valid = false;
        double* ik = info ? info + (size_t)k * UPIC_INFO_COUNT : nullptr;
        rc = s.picard ? picard_one_step(c, s, ik) : implicit_one_step(c, s, ik);
        if (rc) return rc;
        c->steps = s.steps;
        if (diag || step_diag) {
            double* r = diag ? diag + (size_t)k * UPIC_P3_DIAG_COUNT : row;
            if ((rc = state_diagnostics(c, s, r))) return rc;
            s.energy_W = r[UPIC_P3_FIELD_ENERGY];
            s.energy_K = r[UPIC_P3_KINETIC_ENERGY];
            s.energy_valid = true;
        }
        if (step_diag && (rc = step_diagnostics(c, s, W0, K0, s.energy_W, s.energy_K,
                                                step_diag + (size_t)k * UPIC_SD_COUNT)))
            return rc;
    }
    return UPIC_OK;
}

extern "C" const char* upic_convergence_method_name(int code) {
    static const char* const bases[7] = {"none",
                                         "picard",
                                         "picard_fallback",
                                         "current_anderson",
                                         "current_anderson_backtracked",
                                         "current_picard",
                                         "current_picard_backtracked"};
    static const char* const forms[3] = {"", "nested_full_dt_", "selective_"};
    static char names[3][7][48];
    static bool built = false;
    if (!built) {
        for (int f = 0; f < 3; ++f)
            for (int b = 0; b < 7; ++b) std::snprintf(names[f][b], sizeof(names[f][b]), "%s%s", forms[f], bases[b]);
        built = true;
    }
    const int base = code & 7, form = code >> 3;
    if (code < 0 || base > 6 || form > 2) return nullptr;
    return names[form][base];
}

extern "C" int upic_map_log(upic_ctx* c, int capacity, double* rows, int* nrows) {
    if (!c || !nrows || capacity < 0 || (capacity > 0 && !rows)) return c ? fail(c, UPIC_ERR_ARGUMENT, "upic_map_log: bad arguments") : UPIC_ERR_ARGUMENT;
    if (!c->imp) return fail(c, UPIC_ERR_STATE, "context was not created with an implicit method");
    const ImplicitState& s = *c->imp;
    const int n = (int)(s.maplog.size() / UPIC_MAPLOG_COUNT);
    *nrows = n;
    const int k = std::min(n, capacity);
    if (k > 0) std::memcpy(rows, s.maplog.data(), sizeof(double) * UPIC_MAPLOG_COUNT * (size_t)k);
    return UPIC_OK;
}

static_assert(UPIC_FAILLOG_COUNT == 5 + kFailRec, "failed-particle log row = 5 event columns + a record");

extern "C" int upic_failed_particle_log(upic_ctx* c, int capacity, double* rows, int* nrows) {
    if (!c || !nrows || capacity < 0 || (capacity > 0 && !rows))
        return c ? fail(c, UPIC_ERR_ARGUMENT, "upic_failed_particle_log: bad arguments") : UPIC_ERR_ARGUMENT;
    if (!c->imp) return fail(c, UPIC_ERR_STATE, "context was not created with an implicit method");
    const ImplicitState& s = *c->imp;
    const int n = (int)(s.faillog.size() / UPIC_FAILLOG_COUNT);
    *nrows = n;
    const int k = std::min(n, capacity);
    if (k > 0) std::memcpy(rows, s.faillog.data(), sizeof(double) * UPIC_FAILLOG_COUNT * (size_t)k);
    return UPIC_OK;
}

extern "C" int upic_probe_fields(upic_ctx* c, long np, const double* x, const double* y, double* out) {
    if (!c) return UPIC_ERR_ARGUMENT;
    if (!c->imp || c->imp->picard)
        return fail(c, UPIC_ERR_STATE, "upic_probe_fields needs a UPIC_METHOD_CN_ORBIT context");
    ImplicitState& s = *c->imp;
    if (!s.ready) return fail(c, UPIC_ERR_STATE, "upic_init_fields first");
    if (np < 0 || (np > 0 && (!x || !y || !out))) return fail(c, UPIC_ERR_ARGUMENT, "upic_probe_fields: bad arguments");
    if (np == 0) return UPIC_OK;
    for (long p = 0; p < np; ++p)
        if (!std::isfinite(x[p]) || !std::isfinite(y[p])) return fail(c, UPIC_ERR_NONFINITE, "non-finite probe position");
    const int N = c->N;
    int rc;
    if (!s.probe_grid && (rc = dalloc(c, &s.probe_grid, 18 * (size_t)N))) return rc;
    if (np > s.pcap) {
        if ((rc = sync(c))) return rc;
        dfree(c, s.px);
        dfree(c, s.py);
        dfree(c, s.pout);
        s.px = s.py = s.pout = nullptr;
        s.pcap = 0;
        if ((rc = dalloc(c, &s.px, (size_t)np)) || (rc = dalloc(c, &s.py, (size_t)np)) ||
            (rc = dalloc(c, &s.pout, (size_t)np * UPIC_PROBE_COUNT)))
            return rc;
        s.pcap = np;
    }
    // phi, psi, rho, A, U from the state spectra; J; E, B from diag_spectra
    UPIC_CUDA(c, cudaMemcpyAsync(s.dspec, s.spec, sizeof(double2) * 9 * N, cudaMemcpyDeviceToDevice, c->st));
    UPIC_CUDA(c, fft2d_batched(c->plan, s.dspec, 9, 1, c->st, nullptr, 1, s.probe_grid));
    UPIC_CUDA(c, cudaMemcpyAsync(s.probe_grid + 9 * (size_t)N, s.J, sizeof(double) * 3 * N, cudaMemcpyDeviceToDevice,
                                 c->st));
    UPIC_CUDA(c, launch_diag_spectra(N, c->d_kx, c->d_ky, s.spec, s.dspec, c->st));
    UPIC_CUDA(c, fft2d_batched(c->plan, s.dspec, 6, 1, c->st, nullptr, 1, s.probe_grid + 12 * (size_t)N));
    UPIC_CUDA(c, cudaMemcpyAsync(s.px, x, sizeof(double) * np, cudaMemcpyHostToDevice, c->st));
    UPIC_CUDA(c, cudaMemcpyAsync(s.py, y, sizeof(double) * np, cudaMemcpyHostToDevice, c->st));
    UPIC_CUDA(c, launch_probe(s.order, c->nx, c->ny, c->cfg.Lx, c->cfg.Ly, s.probe_grid, np, s.px, s.py, s.pout,
                              c->st));
    UPIC_CUDA(c, cudaMemcpyAsync(out, s.pout, sizeof(double) * UPIC_PROBE_COUNT * np, cudaMemcpyDeviceToHost, c->st));
    return sync(c);
}

extern "C" int upic_set_time_step(upic_ctx* c, double dt) {
    if (!c) return UPIC_ERR_ARGUMENT;
    if (!c->imp) return fail(c, UPIC_ERR_STATE, "upic_set_time_step needs an implicit method");
    if (!std::isfinite(dt) || !(dt > 0.0) || dt > c->imp->dt_max)
        return fail(c, UPIC_ERR_ARGUMENT, "upic_set_time_step: dt must satisfy 0 < dt <= the dt of upic_create");
    c->cfg.dt = dt;
    return UPIC_OK;
}

extern "C" int upic_set_initial_potential(upic_ctx* c, const double* A, const double* U) {
    if (!c) return UPIC_ERR_ARGUMENT;
    if (!c->imp) return fail(c, UPIC_ERR_STATE, "an initial potential needs an implicit method");
    ImplicitState& s = *c->imp;
    if (!A && !U) {
        s.init_AU_set = false;
        return UPIC_OK;
    }
    if (!A || !U) return fail(c, UPIC_ERR_ARGUMENT, "A and U are both needed");
    if (s.picard) return fail(c, UPIC_ERR_STATE, "the non-relativistic method starts from A = U = 0");
    const int N = c->N;
    int rc;
    if (!s.init_AU && (rc = dalloc(c, &s.init_AU, 6 * (size_t)N))) return rc;
    for (long k = 0; k < 3L * N; ++k)
        if (!std::isfinite(A[k]) || !std::isfinite(U[k])) return fail(c, UPIC_ERR_NONFINITE, "non-finite A or U");
    UPIC_CUDA(c, cudaMemcpyAsync(s.init_AU, A, sizeof(double) * 3 * N, cudaMemcpyHostToDevice, c->st));
    UPIC_CUDA(c, cudaMemcpyAsync(s.init_AU + 3 * (size_t)N, U, sizeof(double) * 3 * N, cudaMemcpyHostToDevice,
                                 c->st));
    if ((rc = sync(c))) return rc;
    s.init_AU_set = true;
    return UPIC_OK;
}

// write_field_grid_header / write_field_grid_snapshot (:8137-8140, :8160):
// one row per node, x-major, with the coordinates of Project3's box
// [-L/2, L/2) and every value at 17 significant digits.
extern "C" int upic_write_field_snapshot(upic_ctx* c, const char* path, int append, long step, double time) {
    if (!c || !path) return UPIC_ERR_ARGUMENT;
    if (!c->imp) return fail(c, UPIC_ERR_STATE, "field snapshots carry psi and U: implicit methods only");
    if (!c->imp->ready) return fail(c, UPIC_ERR_STATE, "upic_init_fields first");
    // column order of the snapshot after the coordinates
    static const int kCols[18] = {UPIC_FIELD_PHI, UPIC_FIELD_PSI, UPIC_FIELD_RHO, UPIC_FIELD_AX, UPIC_FIELD_AY,
                                  UPIC_FIELD_AZ,  UPIC_FIELD_UX,  UPIC_FIELD_UY,  UPIC_FIELD_UZ, UPIC_FIELD_JX,
                                  UPIC_FIELD_JY,  UPIC_FIELD_JZ,  UPIC_FIELD_EX,  UPIC_FIELD_EY, UPIC_FIELD_EZ,
                                  UPIC_FIELD_BX,  UPIC_FIELD_BY,  UPIC_FIELD_BZ};
    const int N = c->N;
    std::vector<double> f((size_t)18 * N);
    for (int k = 0; k < 18; ++k) {
        const int rc = implicit_get_field(c, kCols[k], f.data() + (size_t)k * N);
        if (rc) return rc;
    }
    FILE* out = std::fopen(path, append ? "a" : "w");
    if (!out) return fail(c, UPIC_ERR_ARGUMENT, std::string("cannot open ") + path);
    if (!append)
        std::fputs("step,time,spline_order,ix,iy,iz,x,y,z,phi,psi,rho,"
                   "Ax,Ay,Az,Ux,Uy,Uz,Jx,Jy,Jz,Ex,Ey,Ez,Bx,By,Bz\n",
                   out);
    const upic_config& cf = c->cfg;
    const double hx = cf.Lx / c->nx, hy = cf.Ly / c->ny;
    const double z = -0.5 * cf.Lz;
    std::string line;
    char buf[64];
    for (int i = 0; i < c->nx; ++i) {
        for (int j = 0; j < c->ny; ++j) {
            const int id = i * c->ny + j;
            line.clear();
            std::snprintf(buf, sizeof(buf), "%ld,%.17g,%d,%d,%d,0,", step, time, cf.spline_order, i, j);
            line += buf;
            const double xy[3] = {-0.5 * cf.Lx + (double)i * hx, -0.5 * cf.Ly + (double)j * hy, z};
            for (double v : xy) {
                std::snprintf(buf, sizeof(buf), "%.17g,", v);
                line += buf;
            }
            for (int k = 0; k < 18; ++k) {
                std::snprintf(buf, sizeof(buf), k < 17 ? "%.17g," : "%.17g\n", f[(size_t)k * N + id]);
                line += buf;
            }
            std::fputs(line.c_str(), out);
        }
    }
    const bool ok = std::fclose(out) == 0;
    return ok ? UPIC_OK : fail(c, UPIC_ERR_ARGUMENT, std::string("write failed: ") + path);
}

// ---- kernel-level GM-HC push and CN field update -------------------------------

extern "C" int upic_push_gmhc(upic_ctx* c, long np, const double* x, const double* y, const double* P,
                              const double* v, const double* q, const double* m, const double* grad_phi_mid,
                              const double* An, const double* Anp1, double* x1, double* y1, double* P_end,
                              double* v_end, double* vbar, int* report) {
    if (!c) return UPIC_ERR_ARGUMENT;
    if (!c->imp || c->imp->picard)
        return fail(c, UPIC_ERR_STATE, "upic_push_gmhc needs a UPIC_METHOD_CN_ORBIT context");
    if (np < 0 || !grad_phi_mid || !An || !Anp1 ||
        (np > 0 && (!x || !y || !P || !v || !q || !m || !x1 || !y1 || !P_end || !v_end || !vbar || !report)))
        return fail(c, UPIC_ERR_ARGUMENT, "upic_push_gmhc: null array or negative particle count");
    if (np == 0) return UPIC_OK;
    for (long p = 0; p < np; ++p)
        if (!std::isfinite(x[p]) || !std::isfinite(y[p]) || !(m[p] > 0.0) || !std::isfinite(q[p]))
            return fail(c, UPIC_ERR_NONFINITE, "upic_push_gmhc: non-finite position or charge, or mass <= 0");
    ImplicitState& s = *c->imp;
    const upic_config& cf = c->cfg;
    const int N = c->N;
    // node records: grad phi_mid (2), A^n (3), A^{n+1} (3)
    std::vector<double> rec((size_t)kIRec * N), in7(7 * (size_t)np), g3(3 * (size_t)np);
    for (int i = 0; i < N; ++i) {
        double* r = &rec[(size_t)kIRec * i];
        r[kIRecGpm] = grad_phi_mid[i];
        r[kIRecGpm + 1] = grad_phi_mid[N + i];
        for (int k = 0; k < 3; ++k) {
            r[kIRecAn + k] = An[(size_t)k * N + i];
            r[kIRecAe + k] = Anp1[(size_t)k * N + i];
        }
    }
    for (long p = 0; p < np; ++p) {
        in7[p] = x[p];
        in7[np + p] = y[p];
        for (int k = 0; k < 3; ++k) {
            in7[(2 + k) * np + p] = P[3 * p + k];
            g3[k * np + p] = v[3 * p + k];
        }
        in7[5 * np + p] = q[p];
        in7[6 * np + p] = m[p];
    }
    Scratch sc;
    double* drec = sc.get<double>(rec.size());
    double* din = sc.get<double>(in7.size());
    double* dg = sc.get<double>(g3.size());
    double* dout = sc.get<double>(11 * (size_t)np);
    int* drep = sc.get<int>(2 * (size_t)np);
    if (!drec || !din || !dg || !dout || !drep) return fail(c, UPIC_ERR_NOMEM, "upic_push_gmhc: device allocation failed");
    UPIC_CUDA(c, cudaMemcpyAsync(drec, rec.data(), sizeof(double) * rec.size(), cudaMemcpyHostToDevice, c->st));
    UPIC_CUDA(c, cudaMemcpyAsync(din, in7.data(), sizeof(double) * in7.size(), cudaMemcpyHostToDevice, c->st));
    UPIC_CUDA(c, cudaMemcpyAsync(dg, g3.data(), sizeof(double) * g3.size(), cudaMemcpyHostToDevice, c->st));
    ImplicitMapArgs a{};
    a.rec = drec;
    a.Lx = cf.Lx;
    a.Ly = cf.Ly;
    a.inv_dx = 1.0 / s.dx;
    a.inv_dy = 1.0 / s.dy;
    a.dt = cf.dt;
    a.kappa = cf.kappa;
    a.split = cf.split_orbit_at_knots;
    a.loc_rtol = cf.local_rtol;
    a.loc_atol = cf.local_atol;
    a.loc_damp = cf.local_damping;
    a.loc_maxit = cf.local_max_iter;
    a.qtab = s.qtab;
    a.nq = s.nq;
    a.mnq = s.mnq;
    UPIC_CUDA(c, launch_gmhc_push(s.order, a, c->nx, c->ny, np, din, dg, dout, drep, c->st));
    std::vector<double> out(11 * (size_t)np);
    UPIC_CUDA(c, cudaMemcpyAsync(out.data(), dout, sizeof(double) * out.size(), cudaMemcpyDeviceToHost, c->st));
    UPIC_CUDA(c, cudaMemcpyAsync(report, drep, sizeof(int) * 2 * np, cudaMemcpyDeviceToHost, c->st));
    int rc;
    if ((rc = sync(c))) return rc;
    for (long p = 0; p < np; ++p) {
        x1[p] = out[p];
        y1[p] = out[np + p];
        for (int k = 0; k < 3; ++k) {
            P_end[3 * p + k] = out[(2 + k) * np + p];
            v_end[3 * p + k] = out[(5 + k) * np + p];
            vbar[3 * p + k] = out[(8 + k) * np + p];
        }
    }
    return UPIC_OK;
}

extern "C" int upic_fft_solve_cn(upic_ctx* c, const double* phi, const double* psi, const double* rho,
                                 const double* A, const double* U, const double* J, double* phi1, double* psi1,
                                 double* rho1, double* A1, double* U1, double* grad_phi_mid) {
    if (!c) return UPIC_ERR_ARGUMENT;
    if (!c->imp || c->imp->picard)
        return fail(c, UPIC_ERR_STATE, "upic_fft_solve_cn needs a UPIC_METHOD_CN_ORBIT context");
    if (!phi || !psi || !rho || !A || !U || !J || !phi1 || !psi1 || !rho1 || !A1 || !U1)
        return fail(c, UPIC_ERR_ARGUMENT, "upic_fft_solve_cn: null array");
    ImplicitState& s = *c->imp;
    const upic_config& cf = c->cfg;
    const int N = c->N;
    const size_t n = (size_t)N;
    Scratch sc;
    double* dreal = sc.get<double>(9 * n);
    double* dj = sc.get<double>(3 * n);
    double2* sin_ = sc.get<double2>(9 * n);
    double2* sout = sc.get<double2>(9 * n);
    double2* jhat = sc.get<double2>(3 * n);
    double2* gsp = sc.get<double2>(5 * n);
    if (!dreal || !dj || !sin_ || !sout || !jhat || !gsp)
        return fail(c, UPIC_ERR_NOMEM, "upic_fft_solve_cn: device allocation failed");
    // state spectra in the order phi, psi, rho, A (3), U (3)
    const double* src[5] = {phi, psi, rho, A, U};
    const size_t cnt[5] = {n, n, n, 3 * n, 3 * n};
    size_t off = 0;
    for (int k = 0; k < 5; ++k) {
        UPIC_CUDA(c, cudaMemcpyAsync(dreal + off, src[k], sizeof(double) * cnt[k], cudaMemcpyHostToDevice, c->st));
        off += cnt[k];
    }
    UPIC_CUDA(c, fft2d_batched(c->plan, sin_, 9, 0, c->st, dreal));
    // J_field: the Nyquist-projected current (:5265-5266)
    UPIC_CUDA(c, cudaMemcpyAsync(dj, J, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, c->st));
    if (cf.nyquist_projection) UPIC_CUDA(c, launch_project_nyquist(dj, 3, c->nx, c->ny, c->st));
    UPIC_CUDA(c, fft2d_batched(c->plan, jhat, 3, 0, c->st, dj));
    CnArgs k{};
    k.nx = c->nx;
    k.ny = c->ny;
    k.N = N;
    k.kx = c->d_kx;
    k.ky = c->d_ky;
    k.k2 = c->d_k2;
    k.excl = cf.nyquist_projection ? s.excl : nullptr;
    k.Jhat = jhat;
    k.st = sin_;
    k.out = sout;
    k.gspec = gsp;
    k.dt = cf.dt;
    k.kappa = cf.kappa;
    k.sigma1 = cf.sigma1;
    k.sigma2 = cf.sigma2;
    UPIC_CUDA(c, launch_cn_kspace(k, c->st));
    UPIC_CUDA(c, fft2d_batched(c->plan, sout, 9, 1, c->st, nullptr, 1, dreal));
    double* dst[5] = {phi1, psi1, rho1, A1, U1};
    off = 0;
    for (int q = 0; q < 5; ++q) {
        UPIC_CUDA(c, cudaMemcpyAsync(dst[q], dreal + off, sizeof(double) * cnt[q], cudaMemcpyDeviceToHost, c->st));
        off += cnt[q];
    }
    if (grad_phi_mid) {
        int rc;
        if ((rc = sync(c))) return rc;
        UPIC_CUDA(c, fft2d_batched(c->plan, gsp, 2, 1, c->st, nullptr, 1, dreal));
        UPIC_CUDA(c, cudaMemcpyAsync(grad_phi_mid, dreal, sizeof(double) * 2 * n, cudaMemcpyDeviceToHost, c->st));
    }
    return sync(c);
}
