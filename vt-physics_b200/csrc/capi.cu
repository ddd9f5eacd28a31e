// C ABI (include/vtp.h) and the solver driver: config parsing with the
// reference's JSON keys, object attachment in attach order, device state in
// cell-sorted float4 SoA, and one CUDA graph per substep (with conditional
// WHILE nodes for the DFSPH pressure-solve loops).
#include <cmath>
#include <cstdio>
#include <cstring>
#include <algorithm>
#include <memory>
#include <numeric>
#include <string>
#include <vector>

#include <nlohmann/json.hpp>

#include "../../include/vtp.h"
#include "immct.h"
#include "solver.h"

using json = nlohmann::json;

namespace vtp {
thread_local std::string g_last_error;
bool &pdl_flag() {
    static thread_local bool on = false;
    return on;
}
int fail(int code, const std::string &msg) {
    g_last_error = msg;
    return code;
}
}  // namespace vtp

using vtp::fail;
using vtp::g_last_error;

namespace {

#define CU(call)                                                                      \
    do {                                                                              \
        cudaError_t e_ = (call);                                                      \
        if (e_ != cudaSuccess)                                                        \
            return fail(VTP_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

const std::vector<std::string> kPbfRequired = {"animationTime", "timeStep", "particleRadius", "simSpaceLB",
                                               "simSpaceSize", "maxNeighborNum", "iterationNum", "XSPH_k",
                                               "fPartRestDensity", "bPartRestDensity"};
const std::vector<std::string> kDfsphRequired = {"animationTime", "timeStep", "particleRadius", "simSpaceLB",
                                                 "simSpaceSize", "maxNeighborNum", "fPartRestDensity",
                                                 "bPartRestDensity", "fPartRestViscosity", "divFreeThreshold",
                                                 "incompThreshold", "surfaceTensionCoefficient"};
const std::vector<std::string> kObjRequired = {"solverType", "exportFlag", "velocityStart", "colorStart"};
const std::vector<std::string> kOptional = {"enable", "gravity"};

const char *solver_key(int type) {
    switch (type) {
        case VTP_SOLVER_PBF: return "PBF";
        case VTP_SOLVER_DFSPH: return "DFSPH";
        case VTP_SOLVER_IMM: return "IMM";
        case VTP_SOLVER_IMMCT: return "IMMCT";
    }
    return "?";
}

json default_config(int type) {
    json exp = {{"Common", {{"exportTargetDir", "path/to/output"}, {"exportFilePrefix", "obj"},
                            {"exportFileType", "PLY"}}},
                {"SolverRequired", {{"enable", false}, {"exportFps", 35}, {"exportGroupPolicy", "MERGE"}}}};
    json opt = {{"enable", false}, {"gravity", {0, -9.81, 0}}};
    json req;
    if (type == VTP_SOLVER_PBF) {
        req = {{"animationTime", 10}, {"timeStep", 0.01}, {"particleRadius", 0.075},
               {"simSpaceLB", {-1, -1, -1}}, {"simSpaceSize", {2, 2, 2}}, {"maxNeighborNum", 60},
               {"iterationNum", 10}, {"XSPH_k", 0.02}, {"fPartRestDensity", 1000}, {"bPartRestDensity", 1000}};
    } else if (type == VTP_SOLVER_DFSPH) {
        req = {{"animationTime", 10}, {"timeStep", 0.01}, {"particleRadius", 0.075},
               {"simSpaceLB", {-1, -1, -1}}, {"simSpaceSize", {2, 2, 2}}, {"maxNeighborNum", 60},
               {"fPartRestDensity", 1000}, {"bPartRestDensity", 1000}, {"fPartRestViscosity", 0.001},
               {"divFreeThreshold", 1e-4}, {"incompThreshold", 1e-4}, {"surfaceTensionCoefficient", 0.001}};
    } else {
        req = immct_default_required(type == VTP_SOLVER_IMMCT);
    }
    return {{solver_key(type), {{"Required", req}, {"Optional", opt}}}, {"EXPORT", exp}};
}

// Wraps a launch with profiler events when per-kernel timing is active.
#define PROF(self, name, call)                        \
    do {                                              \
        if ((self)->prof) (self)->prof->begin();      \
        call;                                         \
        if ((self)->prof) (self)->prof->end_(name);   \
    } while (0)

// Largest float d2 whose correctly rounded sqrt is <= h.
float sqrt_threshold(float h) {
    float t = h * h;
    while (std::sqrt(t) > h) t = std::nextafter(t, 0.f);
    for (;;) {
        float u = std::nextafter(t, INFINITY);
        if (std::sqrt(u) <= h) t = u;
        else break;
    }
    return t;
}

}  // namespace

// ---------------------------------------------------------------- config

int vtp_solver::parse_config(const json &c) {
    const char *key = solver_key(type);
    if (c.is_null() || c.empty()) return fail(VTP_ERR_CONFIG, std::string(key) + " config json is empty.");
    if (!c.contains(key)) return fail(VTP_ERR_CONFIG, std::string(key) + " config missing main domain: " + key);
    const json &sc = c[key];
    if (!sc.contains("Required"))
        return fail(VTP_ERR_CONFIG, std::string(key) + " config missing necessary domain: Required");
    std::vector<std::string> required;
    if (type == VTP_SOLVER_PBF) required = kPbfRequired;
    else if (type == VTP_SOLVER_DFSPH) required = kDfsphRequired;
    else required = immct_required_keys(type == VTP_SOLVER_IMMCT);
    for (auto &k : required)
        if (!sc["Required"].contains(k))
            return fail(VTP_ERR_CONFIG, std::string(key) + " config missing Required key: " + k);
    if (!sc.contains("Optional")) return fail(VTP_ERR_CONFIG, std::string(key) + " config missing Optional");
    for (auto &k : kOptional)
        if (!sc["Optional"].contains(k))
            return fail(VTP_ERR_CONFIG, std::string(key) + " config missing Optional key: " + k);
    try {
        const json &r = sc["Required"];
        dt = r["timeStep"].get<float>();
        inv_dt = 1.f / dt;
        inv_dt2 = inv_dt * inv_dt;
        radius = r["particleRadius"].get<float>();
        anim_time = r["animationTime"].get<float>();
        auto lb = r["simSpaceLB"].get<std::vector<float>>();
        auto size = r["simSpaceSize"].get<std::vector<float>>();
        if (lb.size() != 3 || size.size() != 3) return fail(VTP_ERR_CONFIG, "simSpaceLB/simSpaceSize need 3 values");
        lbx = lb[0]; lby = lb[1]; lbz = lb[2];
        sx = size[0]; sy = size[1]; sz = size[2];
        maxnbr = r["maxNeighborNum"].get<uint32_t>();
        if (maxnbr < 1 || maxnbr > 1024) return fail(VTP_ERR_CONFIG, "maxNeighborNum must be in [1, 1024]");
        // h = 4 r, rest volume (2r)^3 (PBFSolver.cpp:50-51).
        h = radius * 4;
        vol0 = std::pow(2 * radius, 3.f);
        gravity = make_float3(0.f, -9.8f, 0.f);
        if (sc["Optional"]["enable"].get<bool>()) {
            auto g = sc["Optional"]["gravity"].get<std::vector<float>>();
            if (g.size() != 3) return fail(VTP_ERR_CONFIG, "gravity needs 3 values");
            gravity = make_float3(g[0], g[1], g[2]);
        }
        if (type == VTP_SOLVER_PBF) {
            rho_f = r["fPartRestDensity"].get<float>();
            rho_b = r["bPartRestDensity"].get<float>();
            iterations = r["iterationNum"].get<int>();
            xsph_k = r["XSPH_k"].get<float>();
        } else if (type == VTP_SOLVER_DFSPH) {
            rho_f = r["fPartRestDensity"].get<float>();
            rho_b = r["bPartRestDensity"].get<float>();
            viscosity = r["fPartRestViscosity"].get<float>();
            div_thr = r["divFreeThreshold"].get<float>();
            incomp_thr = r["incompThreshold"].get<float>();
            gamma = r["surfaceTensionCoefficient"].get<float>();
        } else {
            int rc = immct_parse(type == VTP_SOLVER_IMMCT, r, imm);
            if (rc) return rc;
            rho_b = 0.f;   // IMM / IMM-CT boundaries carry volume only
            div_thr = r["divFreeThreshold"].get<float>();
            incomp_thr = r["incompThreshold"].get<float>();
            gamma = r["surfaceTensionCoefficient"].get<float>();
        }
        // extension defaults (a config without a "B200" block restores them)
        force_div = force_inc = 0;
        force_seq.clear();
        device_loop = true; use_graphs = true; stage_timers = false; stop_on_crash = true;
        block = 128; unroll = 4; persistent_tiles = false; cube_powf = false; list_lanes = 0; row_lanes = 1;
        cell_cull = false; staged_solve = false; stage_rows = 2048; tape_budget_mb = 8192; adj_lanes = 1;
        cfl = 0.f;
        cell_order_brick = true;
        pbf_form = 0; pbf_eps = 1e-6f;
        if (c.contains("B200")) {
            const json &b = c["B200"];
            force_div = b.value("forceDivIterations", 0u);
            force_inc = b.value("forceIncompIterations", 0u);
            force_seq.clear();
            if (b.contains("forceIterationsPerTick")) {
                for (auto &pair : b["forceIterationsPerTick"]) {
                    auto v = pair.get<std::vector<uint32_t>>();
                    if (v.size() != 2) return fail(VTP_ERR_CONFIG, "forceIterationsPerTick entries are [div, incomp]");
                    force_seq.push_back(v[0]);
                    force_seq.push_back(v[1]);
                }
            }
            device_loop = b.value("deviceLoop", true);
            use_graphs = b.value("useGraphs", true);
            stage_timers = b.value("stageTimers", false);
            stop_on_crash = b.value("stopOnNonConvergence", true);
            block = b.value("blockSize", 128);
            unroll = b.value("unroll", 4);
            persistent_tiles = b.value("persistentTiles", false);
            cfl = b.value("cfl", 0.f);
            if (!(cfl >= 0.f && cfl <= 1.f)) return fail(VTP_ERR_CONFIG, "cfl must be in [0, 1] (0: fixed timeStep)");
            if (cfl > 0.f && type != VTP_SOLVER_DFSPH)
                return fail(VTP_ERR_CONFIG, "cfl (adaptive time step) is a DFSPH extension");
            const std::string order = b.value("cellOrder", std::string("brick"));
            if (order != "brick" && order != "linear")
                return fail(VTP_ERR_CONFIG, "cellOrder must be \"brick\" or \"linear\"");
            cell_order_brick = order == "brick";
            pdl = b.value("pdl", true);
            row_lanes = b.value("rowLanes", 1);
            if (row_lanes != 1 && row_lanes != 4 && row_lanes != 8)
                return fail(VTP_ERR_CONFIG, "rowLanes must be 1, 4 or 8");
            cell_cull = b.value("cellCull", false);
            staged_solve = b.value("stagedSolve", false);
            tape_budget_mb = b.value("tapeBudgetMB", 8192u);
            adj_lanes = b.value("adjointLanes", 1);
            if (adj_lanes != 1 && adj_lanes != 2 && adj_lanes != 4 && adj_lanes != 8)
                return fail(VTP_ERR_CONFIG, "adjointLanes must be 1, 2, 4 or 8");
            stage_rows = b.value("stageRows", 2048);
            if (stage_rows < 256 || stage_rows > (int)vtp::kStageMaxRows)
                return fail(VTP_ERR_CONFIG, "stageRows must be in [256, 32767]");
            list_lanes = b.value("listLanes", 0);
            if (list_lanes != 0 && list_lanes != 1 && list_lanes != 8)
                return fail(VTP_ERR_CONFIG, "listLanes must be 0 (by row count), 1 or 8");
            const std::string cube = b.value("cubicCube", std::string("rounded"));
            if (cube != "rounded" && cube != "powf")
                return fail(VTP_ERR_CONFIG, "cubicCube must be \"rounded\" or \"powf\"");
            cube_powf = cube == "powf";
            const std::string retry = b.value("phaseRetry", std::string("nearFlagged"));
            if (retry != "nearFlagged" && retry != "all")
                return fail(VTP_ERR_CONFIG, "phaseRetry must be \"nearFlagged\" or \"all\"");
            phase_retry_all = retry == "all";
            const std::string form = b.value("pbfFormulation", std::string("reference"));
            if (form != "reference" && form != "standard")
                return fail(VTP_ERR_CONFIG, "pbfFormulation must be \"reference\" or \"standard\"");
            pbf_form = form == "standard" ? 1 : 0;
            pbf_eps = b.value("pbfEpsilon", pbf_form ? 100.f : 1e-6f);
            if (unroll != 1 && unroll != 2 && unroll != 4 && unroll != 8)
                return fail(VTP_ERR_CONFIG, "unroll must be 1, 2, 4 or 8");
            if (block < 32 || block > 256 || (block & 31)) return fail(VTP_ERR_CONFIG, "blockSize must be 32..256, multiple of 32");
        }
    } catch (const std::exception &e) {
        return fail(VTP_ERR_CONFIG, std::string("config value error: ") + e.what());
    }
    // EXPORT block (optional here; the reference's templates always carry it)
    export_enabled = false;
    if (c.contains("EXPORT")) {
        try {
            const json &ex = c["EXPORT"];
            export_enabled = ex.at("SolverRequired").at("enable").get<bool>();
            if (export_enabled) {
                const float fps = ex.at("SolverRequired").at("exportFps").get<float>();
                if (!(fps > 0.f)) return fail(VTP_ERR_CONFIG, "exportFps must be > 0");
                export_gap = 1.f / fps;
                for (const char *k : {"exportTargetDir", "exportFilePrefix"})
                    if (!ex.at("Common").contains(k)) return fail(VTP_ERR_CONFIG, std::string("Export Common Config missing key: ") + k);
                if (!ex.at("SolverRequired").contains("exportGroupPolicy"))
                    return fail(VTP_ERR_CONFIG, "Export SolverRequired Config missing key: exportGroupPolicy");
            }
        } catch (const std::exception &e) {
            return fail(VTP_ERR_CONFIG, std::string("EXPORT config error: ") + e.what());
        }
    }
    cfg = c;
    configured = true;
    // setConfig (re)defines scene 0 and drops any added scenes.
    SceneRec s0;
    s0.lb[0] = lbx; s0.lb[1] = lby; s0.lb[2] = lbz;
    s0.size[0] = sx; s0.size[1] = sy; s0.size[2] = sz;
    s0.gravity = gravity;
    scenes.assign(1, s0);
    return VTP_OK;
}

int vtp_solver::add_scene(const json &c, uint32_t *index) {
    if (!configured) return fail(VTP_ERR_STATE, "add_scene before setConfig");
    if (initialized) return fail(VTP_ERR_STATE, "add_scene after initialize");
    if (type != VTP_SOLVER_PBF && type != VTP_SOLVER_DFSPH)
        return fail(VTP_ERR_CONFIG, "scene batching supports the PBF and DFSPH solvers");
    if (scenes.size() >= 65535) return fail(VTP_ERR_BOUNDS, "too many scenes");
    // Parse with a scratch solver, then require every shared parameter to match.
    vtp_solver t;
    t.type = type;
    int rc = t.parse_config(c);
    if (rc) return rc;
    std::string diff;
    auto same = [&](const char *name, double a, double b) {
        if (a != b && diff.empty()) diff = name;
    };
    same("timeStep", t.dt, dt);
    same("particleRadius", t.radius, radius);
    same("maxNeighborNum", t.maxnbr, maxnbr);
    same("fPartRestDensity", t.rho_f, rho_f);
    same("bPartRestDensity", t.rho_b, rho_b);
    same("iterationNum", t.iterations, iterations);
    same("XSPH_k", t.xsph_k, xsph_k);
    same("fPartRestViscosity", t.viscosity, viscosity);
    same("divFreeThreshold", t.div_thr, div_thr);
    same("incompThreshold", t.incomp_thr, incomp_thr);
    same("surfaceTensionCoefficient", t.gamma, gamma);
    if (!diff.empty())
        return fail(VTP_ERR_CONFIG, "scene config differs from scene 0 in a shared parameter: " + diff);
    scenes.push_back(t.scenes[0]);
    if (index) *index = (uint32_t)(scenes.size() - 1);
    return VTP_OK;
}

int vtp_solver::attach(const float *p, uint32_t n, const float *v, const json &o) {
    if (initialized) return fail(VTP_ERR_STATE, "attach after initialize");
    json occ = o.value("ObjectComponentConfig", json::object());
    json socc = o.value("SolverObjectComponentConfig", json::object());
    if (!occ.contains("epmMaterial")) return fail(VTP_ERR_CONFIG, "object has no epmMaterial");
    int mat = occ["epmMaterial"].get<int>();
    if (mat != 0 && mat != 1) return fail(VTP_ERR_CONFIG, std::string(solver_key(type)) + "Solver unsupported material.");
    const bool mix = type == VTP_SOLVER_IMM || type == VTP_SOLVER_IMMCT;
    static const std::vector<std::string> kMixObjRequired = {"solverType", "exportFlag", "velocityStart",
                                                             "phaseFraction"};
    for (auto &k : (mix ? kMixObjRequired : kObjRequired))
        if (!socc.contains(k))
            return fail(VTP_ERR_CONFIG, "Object has no " + std::string(solver_key(type)) + " object component config key: " + k);
    if (socc["solverType"].get<int>() != type)
        return fail(VTP_ERR_CONFIG, std::string("Object has no ") + solver_key(type) + " object component config.");
    if (n > 0 && !p) return fail(VTP_ERR_ARG, "null positions");
    ObjRec rec;
    rec.name = o.value("name", std::string("obj_") + std::to_string(objs.size()));
    rec.mat = mat;
    rec.scene = o.value("scene", 0u);
    if (rec.scene >= scenes.size()) return fail(VTP_ERR_ARG, "object scene index out of range");
    rec.start = (uint32_t)(hpos.size() / 3);
    rec.export_flag = socc["exportFlag"].get<bool>();
    auto v0 = socc["velocityStart"].get<std::vector<float>>();
    auto c0 = socc.value("colorStart", std::vector<float>{0.f, 0.f, 0.f});
    for (int a = 0; a < 3; ++a) {
        rec.vel0[a] = a < (int)v0.size() ? v0[a] : 0.f;
        rec.color[a] = a < (int)c0.size() ? c0[a] : 0.f;
    }
    if (mix) {
        rec.phase = socc["phaseFraction"].get<std::vector<float>>();
        if (!imm || (int)rec.phase.size() != immct_phase_count(*this))
            return fail(VTP_ERR_CONFIG, "Object phaseFraction size not match with solver.");
    }
    hpos.insert(hpos.end(), p, p + 3 * (size_t)n);
    for (uint32_t i = 0; i < n; ++i)
        for (int a = 0; a < 3; ++a) {
            hvel.push_back(v ? v[3 * (size_t)i + a] : rec.vel0[a]);
            hcolor.push_back(rec.color[a]);
        }
    hmat.insert(hmat.end(), n, mat);
    if (!rec.phase.empty())
        for (uint32_t i = 0; i < n; ++i) hphase.insert(hphase.end(), rec.phase.begin(), rec.phase.end());
    rec.end = (uint32_t)(hpos.size() / 3);
    objs.push_back(rec);
    return VTP_OK;
}

// ---------------------------------------------------------------- args

vtp::PbfArgs vtp_solver::pbf_args() {
    vtp::PbfArgs a{};
    a.nf = L.nf; a.nb = L.nb; a.ell_stride = L.ell_stride; a.k = kc;
    a.rho0 = rho_f; a.inv_rho0 = 1.f / rho_f; a.rho_b = rho_b; a.eps = pbf_eps; a.dt = dt; a.xsph_k = xsph_k;
    a.form = pbf_form;
    a.h2 = h * h;
    a.c6 = (float)(315.0 / (64.0 * 3.14159265358979 * std::pow((double)h, 9.0)));
    a.cs = (float)(-45.0 / (3.14159265358979 * std::pow((double)h, 6.0)));
    a.nbr = u.nbr; a.ncnt = u.ncnt;
    a.pos = pos.c(); a.pos_alt = pos.n(); a.vel = vel.c(); a.vel_alt = vel.n();
    a.vol = vol; a.density = density; a.lambda = lambda;
    a.unroll = unroll;
    a.lanes = row_lanes;
    return a;
}

vtp::DfsphArgs vtp_solver::dfsph_args(int which) {
    vtp::DfsphArgs a{};
    a.nf = L.nf; a.nb = L.nb; a.ell_stride = L.ell_stride; a.k = kc;
    a.dt = dt; a.inv_dt = inv_dt; a.inv_dt2 = inv_dt2;
    a.rho0 = rho_f; a.rho_b = rho_b; a.vol_f = vol0;
    a.mass_f = rho_f * vol0;                               // update_mass_cuda: m = rest_density * V
    a.vis_coef = (viscosity + viscosity) / 2 * a.mass_f / rho_f;
    a.h2_001 = 0.001f * (h * h);
    a.gamma = gamma;
    a.csigma = 32.f / 3.14159265f / std::pow(h, 9.f);
    a.h6_64 = std::pow(h, 6.f) / 64;
    a.nbr = u.nbr; a.ncnt = u.ncnt;
    a.pos = pos.c(); a.vel = vel.c(); a.vel_alt = vel.n(); a.vadv = vadv.c(); a.vadv_alt = vadv.n();
    a.ratio = ratio; a.alpha = alpha; a.kappa = kappa; a.delta = delta;
    a.acc_tmp = acc_tmp; a.normal = normal;
    a.orig = orig.c(); a.obj_of = obj_of; a.nobj_max = nobj_max; a.partials = partials; a.status = d_status;
    a.tiles = d_tiles; a.ntiles = ntiles; a.scene_tiles = d_scene_tiles; a.persistent = persistent_tiles;
    a.state = solve ? solve + (size_t)which * scenes.size() : nullptr;
    a.sc = scn();
    a.pva = pva;
    a.pk = pk;
    a.tick = d_tick;
    a.unroll = unroll;
    a.staged = staged ? 1 : 0;
    a.stg = stg;
    a.dtp = cfl > 0.f ? d_cfl : nullptr;
    a.vmax_bits = cfl > 0.f ? d_vmax : nullptr;
    return a;
}

vtp::SolveCtl vtp_solver::solve_ctl(int which, cudaGraphConditionalHandle hnd, int use_cond) {
    vtp::SolveCtl c{};
    c.state = solve + (size_t)which * scenes.size();
    c.loop = loop + which;
    c.inv_count = inv_count;
    c.scene_tiles = staged ? d_scene_groups : d_scene_tiles;
    c.nscenes = nscenes();
    c.nobj_max = nobj_max;
    c.threshold = which == 0 ? div_thr : incomp_thr;
    c.force_iters = which == 0 ? force_div : force_inc;
    c.force_seq = d_force_seq;
    c.force_seq_len = (uint32_t)(force_seq.size() / 2);
    c.tick = d_tick;
    c.which = which;
    c.max_iters = 101;
    c.cond = hnd;
    c.use_cond = use_cond;
    return c;
}

// ---------------------------------------------------------------- initialize

int vtp_solver::sort_boundary_and_lists() {
    // Boundary rows are static: sort them once, build the cell table once.
    vtp::Carry none{};
    vtp::ugns_sort(st, scn(), nbuckets, L.nf, L.nb, pos.c(), pos.n(), vel.c(), vel.n(), orig.c(), orig.n(), none, 0.f,
                   u, u.bstart);
    // Copy the sorted boundary rows into both buffers of every double buffer.
    size_t nb = L.nb;
    CU(cudaMemcpyAsync(pos.c() + L.nf, pos.n() + L.nf, nb * sizeof(float4), cudaMemcpyDeviceToDevice, st));
    CU(cudaMemcpyAsync(vel.c() + L.nf, vel.n() + L.nf, nb * sizeof(float4), cudaMemcpyDeviceToDevice, st));
    CU(cudaMemcpyAsync(orig.c() + L.nf, orig.n() + L.nf, nb * sizeof(uint32_t), cudaMemcpyDeviceToDevice, st));
    return VTP_OK;
}

int vtp_solver::initialize() {
    const vtp::NvtxRange nvtx_range("vtp initialize");
    if (!configured) return fail(VTP_ERR_STATE, "initialize before setConfig");
    if (initialized) return VTP_OK;
    const uint32_t n = (uint32_t)(hpos.size() / 3);
    if (n == 0) return fail(VTP_ERR_STATE, "no particles attached");
    const int S = nscenes();
    if (cfl > 0.f && S != 1)
        return fail(VTP_ERR_CONFIG, "cfl (adaptive time step) needs a single scene: batched scenes share one step");
    L.n = n;
    L.nf = 0;
    for (auto &sc : scenes) sc.nf = sc.nb = 0, sc.attach_lo = UINT32_MAX;
    for (auto &o : objs) {
        SceneRec &sc = scenes[o.scene];
        (o.mat == 0 ? sc.nf : sc.nb) += o.end - o.start;
        if (o.end > o.start) sc.attach_lo = std::min(sc.attach_lo, o.start);
        if (o.mat == 0) L.nf += o.end - o.start;
    }
    L.nb = n - L.nf;
    L.ell_stride = maxnbr > 1 ? maxnbr - 1 : 1;
    // Attach ids of fluid vs boundary decide how a cell's two runs interleave
    // (per scene; scenes that disagree fall back to the general merge).
    int mode = -1;
    for (int k = 0; k < S; ++k) {
        uint32_t fmin = UINT32_MAX, fmax = 0, bmin = UINT32_MAX, bmax = 0;
        for (auto &o : objs) {
            if (o.end == o.start || (int)o.scene != k) continue;
            if (o.mat == 0) fmin = std::min(fmin, o.start), fmax = std::max(fmax, o.end - 1);
            else bmin = std::min(bmin, o.start), bmax = std::max(bmax, o.end - 1);
        }
        int m;
        if (scenes[k].nb == 0 || scenes[k].nf == 0 || fmax < bmin) m = 0;
        else if (bmax < fmin) m = 1;
        else m = 2;
        if (scenes[k].nf + scenes[k].nb == 0) continue;
        mode = mode < 0 ? m : (mode == m ? m : 2);
    }
    L.merge_mode = mode < 0 ? 0 : mode;
    L.list_lanes = list_lanes;
    L.cell_cull = cell_cull;

    // Grids as UniformGirdNeighborSearcher::setConfig (UniformGridNeighborSearch.cpp:214-218),
    // one per scene, each followed by its own outside bucket.
    uint64_t key_base = 0;
    uint32_t fb = 0, bb = L.nf;
    for (auto &sc : scenes) {
        vtp::SceneGrid &g = sc.grid;
        g.lbx = sc.lb[0]; g.lby = sc.lb[1]; g.lbz = sc.lb[2];
        g.gx = (int)std::ceil(sc.size[0] / h);
        g.gy = (int)std::ceil(sc.size[1] / h);
        g.gz = (int)std::ceil(sc.size[2] / h);
        if (g.gx <= 0 || g.gy <= 0 || g.gz <= 0) return fail(VTP_ERR_CONFIG, "empty grid");
        // Cells 0..g per axis (the inclusive upper bound of cellIsAvailable).  Bricked
        // bucket order (4^3-cell bricks, Morton inside) unless the grid is under 4
        // cells wide in x or y; the linear key reaches z*gy*gx + y*gx + x.
        const uint64_t bx = (uint64_t)(g.gx + 4) / 4, by = (uint64_t)(g.gy + 4) / 4,
                       bz = (uint64_t)(g.gz + 4) / 4;
        g.brick = (cell_order_brick && g.gx >= 4 && g.gy >= 4) ? 1 : 0;
        g.bx = (uint32_t)bx;
        g.by = (uint32_t)by;
        uint64_t maxkey = g.brick ? bx * by * bz * 64 - 1
                                  : (uint64_t)g.gz * g.gy * g.gx + (uint64_t)g.gy * g.gx + g.gx;
        if (maxkey + 2 > (1ull << 31)) return fail(VTP_ERR_BOUNDS, "grid too large (more than 2^31 cells)");
        g.nkey = (uint32_t)(maxkey + 1);
        g.key_base = (uint32_t)key_base;
        g.grav_x = sc.gravity.x; g.grav_y = sc.gravity.y; g.grav_z = sc.gravity.z;
        key_base += (uint64_t)g.nkey + 1;
        if (key_base + 1 > (1ull << 31)) return fail(VTP_ERR_BOUNDS, "scene grids too large (more than 2^31 cells)");
        sc.fbase = fb; fb += sc.nf;
        sc.bbase = bb; bb += sc.nb;
    }
    nbuckets = (uint32_t)key_base;
    d2max = sqrt_threshold(h);
    kc.h = h;
    kc.invh = 1.f / h;
    kc.sigma = 8.f / 3.14159265f / std::pow(h, 3.f);  // replaced by the device value below
    kc.w0 = kc.sigma;
    kc.cube_powf = cube_powf ? 1 : 0;

    if (!st) {
        CU(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        CU(cudaStreamCreateWithFlags(&side, cudaStreamNonBlocking));
        CU(cudaStreamCreateWithFlags(&side2, cudaStreamNonBlocking));
        CU(cudaEventCreateWithFlags(&ev_fork, cudaEventDisableTiming));
        CU(cudaEventCreateWithFlags(&ev_join, cudaEventDisableTiming));
        for (auto &e : ev) CU(cudaEventCreate(&e));
        CU(cudaMallocHost((void **)&h_pinned, 8 * sizeof(uint32_t)));
    }
    if (vtp::cubic_sigma_device(st, h, &kc.sigma)) return fail(VTP_ERR_CUDA, "cubic sigma kernel failed");
    kc.w0 = kc.sigma;  // W(0) = sigma * (6*0 - 6*0 + 1)
    int rc;
#define AL(p, cnt) \
    if ((rc = alloc(p, cnt))) return rc
    for (int k = 0; k < 2; ++k) {
        AL(&pos.b[k], n);
        AL(&vel.b[k], n);
        AL(&orig.b[k], n);
    }
    const uint32_t nrows_max = std::max(L.nf, L.nb);
    AL(&u.key, nrows_max);
    AL(&u.rank, nrows_max);
    AL(&u.count, (size_t)nbuckets);
    CU(cudaMemsetAsync(u.count, 0, (size_t)nbuckets * sizeof(uint32_t), st));   // kept zero by the cell scan
    AL(&u.fstart, (size_t)nbuckets + 1);
    AL(&u.bstart, (size_t)nbuckets + 1);
    AL(&u.tmp_src, nrows_max);
    AL(&u.tmp_orig, nrows_max);
    AL(&u.tmp_key, nrows_max);
    u.scan_tiles = ((size_t)nbuckets + 2047) / 2048;
    if (u.scan_tiles > 1024 * 64) return fail(VTP_ERR_BOUNDS, "grid too large for the cell scan");
    AL(&u.scan_sums, u.scan_tiles);
    const size_t fl_rows = ((size_t)L.nf + 31) / 32 * 32, bl_rows = ((size_t)L.nb + 31) / 32 * 32;
    AL(&u.nbr, fl_rows * L.ell_stride);
    AL(&u.ncnt, L.nf);
    AL(&u.bnbr, bl_rows * L.ell_stride);
    AL(&u.bncnt, L.nb);
    AL(&d_status, 4);
    u.status = d_status;
    AL(&d_overflow, 4);
    CU(cudaMemsetAsync(d_status, 0, 4 * sizeof(uint32_t), st));
    CU(cudaMemsetAsync(d_overflow, 0, 4 * sizeof(uint32_t), st));

    // Scene table and the static row -> scene map.
    std::vector<vtp::SceneGrid> sg(S);
    std::vector<uint16_t> rs(n);
    for (int k = 0; k < S; ++k) {
        sg[k] = scenes[k].grid;
        std::fill(rs.begin() + scenes[k].fbase, rs.begin() + scenes[k].fbase + scenes[k].nf, (uint16_t)k);
        std::fill(rs.begin() + scenes[k].bbase, rs.begin() + scenes[k].bbase + scenes[k].nb, (uint16_t)k);
    }
    AL(&d_sg, S);
    AL(&row_scene, n);
    CU(cudaMemcpyAsync(d_sg, sg.data(), S * sizeof(vtp::SceneGrid), cudaMemcpyHostToDevice, st));
    CU(cudaMemcpyAsync(row_scene, rs.data(), n * sizeof(uint16_t), cudaMemcpyHostToDevice, st));

    // Upload in attach order, placing each scene's fluid rows in [fbase, fbase + nf) and its
    // boundary rows in [bbase, bbase + nb), attach order kept inside each range.
    std::vector<float4> p4(n), v4(n);
    std::vector<uint32_t> ids(n);
    std::vector<uint32_t> fnext(S), bnext(S);
    for (int k = 0; k < S; ++k) fnext[k] = scenes[k].fbase, bnext[k] = scenes[k].bbase;
    std::vector<int> scene_of(n, 0);
    for (auto &o : objs)
        for (uint32_t i = o.start; i < o.end; ++i) scene_of[i] = (int)o.scene;
    const float mass_f = rho_f * vol0;
    for (uint32_t i = 0; i < n; ++i) {
        const int k = scene_of[i];
        uint32_t row = hmat[i] == 0 ? fnext[k]++ : bnext[k]++;
        float w = 0.f;
        if (type == VTP_SOLVER_PBF) w = mass_f;          // PBF: w = mass (init_cuda, PBFCudaImpl.cu:34-45)
        else w = vol0;                                    // DFSPH / IMM: w = volume
        p4[row] = make_float4(hpos[3 * i], hpos[3 * i + 1], hpos[3 * i + 2], w);
        v4[row] = make_float4(hvel[3 * i], hvel[3 * i + 1], hvel[3 * i + 2], 0.f);
        ids[row] = i;
    }
    CU(cudaMemcpyAsync(pos.c(), p4.data(), n * sizeof(float4), cudaMemcpyHostToDevice, st));
    CU(cudaMemcpyAsync(vel.c(), v4.data(), n * sizeof(float4), cudaMemcpyHostToDevice, st));
    CU(cudaMemcpyAsync(orig.c(), ids.data(), n * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
    CU(cudaMemcpyAsync(pos.n(), p4.data(), n * sizeof(float4), cudaMemcpyHostToDevice, st));
    CU(cudaMemcpyAsync(vel.n(), v4.data(), n * sizeof(float4), cudaMemcpyHostToDevice, st));
    CU(cudaMemcpyAsync(orig.n(), ids.data(), n * sizeof(uint32_t), cudaMemcpyHostToDevice, st));

    if ((rc = sort_boundary_and_lists())) return rc;

    // Solver-specific buffers.
    if (type == VTP_SOLVER_PBF) {
        AL(&vol, n);
        AL(&density, L.nf);
        AL(&lambda, L.nf);
        std::vector<float> v(n, vol0);
        CU(cudaMemcpyAsync(vol, v.data(), n * sizeof(float), cudaMemcpyHostToDevice, st));
        CU(cudaMemsetAsync(density, 0, std::max<size_t>(L.nf, 1) * sizeof(float), st));
        CU(cudaMemsetAsync(lambda, 0, std::max<size_t>(L.nf, 1) * sizeof(float), st));
    } else {
        for (int k = 0; k < 2; ++k) AL(&vadv.b[k], n);
        AL(&pva, 2 * (size_t)n);
        AL(&pk, n);
        AL(&ratio, L.nf);
        AL(&alpha, L.nf);
        AL(&kappa, L.nf);
        AL(&delta, L.nf);
        AL(&rest_b, L.nb);
        AL(&acc_tmp, L.nf);
        AL(&normal, L.nf);
        AL(&solve, 2 * (size_t)S);
        CU(cudaMemsetAsync(solve, 0, 2 * (size_t)S * sizeof(vtp::SolveState), st));
        AL(&loop, 2);
        CU(cudaMemsetAsync(loop, 0, 2 * sizeof(vtp::LoopState), st));
        AL(&d_tick, 1);
        if (cfl > 0.f) {
            AL(&d_cfl, 2);
            AL(&d_vmax, 1);
            const float init[2] = {dt, 0.f};
            CU(cudaMemcpyAsync(d_cfl, init, sizeof(init), cudaMemcpyHostToDevice, st));
            CU(cudaMemsetAsync(d_vmax, 0, sizeof(uint32_t), st));
        }
        CU(cudaMemsetAsync(d_tick, 0, sizeof(uint64_t), st));
        if (!force_seq.empty()) {
            AL(&d_force_seq, force_seq.size());
            CU(cudaMemcpyAsync(d_force_seq, force_seq.data(), force_seq.size() * sizeof(uint32_t),
                               cudaMemcpyHostToDevice, st));
        }
        CU(cudaMemsetAsync(kappa, 0, std::max<size_t>(L.nf, 1) * sizeof(float), st));
        CU(cudaMemsetAsync(ratio, 0, std::max<size_t>(L.nf, 1) * sizeof(float), st));
        CU(cudaMemsetAsync(alpha, 0, std::max<size_t>(L.nf, 1) * sizeof(float), st));
        CU(cudaMemsetAsync(delta, 0, std::max<size_t>(L.nf, 1) * sizeof(float), st));
        // Fluid objects: residual means are taken per object (vfsph_div, DFSPHCudaImpl.cu:471-483);
        // slots are numbered scene by scene so a scene's objects are contiguous.
        std::vector<uint16_t> objmap(n, 0);
        std::vector<double> invc;
        std::vector<vtp::SceneTiles> stl(S);
        nobj_max = 1;
        for (int k = 0; k < S; ++k) {
            stl[k].obj0 = (uint32_t)invc.size();
            for (auto &o : objs) {
                if (o.mat != 0 || (int)o.scene != k) continue;
                for (uint32_t i = o.start; i < o.end; ++i) objmap[i] = (uint16_t)invc.size();
                invc.push_back(o.end > o.start ? 1.0 / (double)(o.end - o.start) : 0.0);
            }
            stl[k].nobj = (uint32_t)invc.size() - stl[k].obj0;
            nobj_max = std::max<int>(nobj_max, (int)stl[k].nobj);
        }
        if (invc.size() > 65535) return fail(VTP_ERR_BOUNDS, "too many fluid objects");
        if (invc.empty()) invc.push_back(0.0);
        // Scene-offset tiles of `block` fluid rows each.
        std::vector<uint4> tiles;
        for (int k = 0; k < S; ++k) {
            stl[k].tile0 = (uint32_t)tiles.size();
            for (uint32_t r = 0; r < scenes[k].nf; r += (uint32_t)block)
                tiles.push_back(make_uint4(scenes[k].fbase + r, std::min<uint32_t>(block, scenes[k].nf - r),
                                           (uint32_t)k, 0u));
            stl[k].ntiles = (uint32_t)tiles.size() - stl[k].tile0;
        }
        ntiles = (uint32_t)tiles.size();
        AL(&inv_count, invc.size());
        AL(&obj_of, n);
        AL(&d_tiles, std::max<size_t>(tiles.size(), 1));
        AL(&d_tile_ran, std::max<size_t>(tiles.size(), 1));
        AL(&d_scene_tiles, S);
        CU(cudaMemcpyAsync(inv_count, invc.data(), invc.size() * sizeof(double), cudaMemcpyHostToDevice, st));
        CU(cudaMemcpyAsync(obj_of, objmap.data(), n * sizeof(uint16_t), cudaMemcpyHostToDevice, st));
        if (!tiles.empty())
            CU(cudaMemcpyAsync(d_tiles, tiles.data(), tiles.size() * sizeof(uint4), cudaMemcpyHostToDevice, st));
        CU(cudaMemcpyAsync(d_scene_tiles, stl.data(), S * sizeof(vtp::SceneTiles), cudaMemcpyHostToDevice, st));
        // Staged pressure solve: one scene in bricked order whose cells' fluid and boundary runs
        // do not interleave; residual partials per cell group (plus one for the rows outside).
        staged = staged_solve && type == VTP_SOLVER_DFSPH && S == 1 && scenes[0].grid.brick &&
                 L.merge_mode != 2 && L.nf > 0;
        size_t npart = std::max<uint32_t>(ntiles, 1);
        if (staged) {
            stg.ngroups = scenes[0].grid.nkey / vtp::kStageBuckets;
            stg.scap = (uint32_t)stage_rows;
            stg.mode = L.merge_mode;
            stg.fstart = u.fstart;
            stg.bstart = u.bstart;
            const size_t fl_rows = ((size_t)L.nf + 31) / 32 * 32;
            AL(&stg.snbr, fl_rows * L.ell_stride);
            vtp::SceneTiles sg = stl[0];
            sg.tile0 = 0;
            sg.ntiles = stg.ngroups + 1;
            AL(&d_scene_groups, 1);
            CU(cudaMemcpyAsync(d_scene_groups, &sg, sizeof(sg), cudaMemcpyHostToDevice, st));
            npart = std::max<size_t>(npart, (size_t)stg.ngroups + 1);
        }
        AL(&partials, npart * nobj_max + 1);
        if (type != VTP_SOLVER_DFSPH) {
            if ((rc = immct_alloc(*this))) return rc;
        }
    }
    // Neighbour search of the initial state (initialize(): m_neighborSearcher.update(pos)),
    // then the boundary volumes from the boundary rows' lists.
    vtp::Carry carry{};
    vtp::ugns_sort(st, scn(), nbuckets, 0, L.nf, pos.c(), pos.n(), vel.c(), vel.n(), orig.c(), orig.n(), carry, 0.f,
                   u, u.fstart);
    pos.swap(); vel.swap(); orig.swap();
    vtp::ugns_build_lists(st, scn(), L, 0, L.nf, pos.c(), orig.c(), u, u.nbr, u.ncnt, d_status, d_overflow, block);
    vtp::ugns_build_lists(st, scn(), L, L.nf, L.nb, pos.c(), orig.c(), u, u.bnbr, u.bncnt, d_status, d_overflow,
                          block);
    if (type == VTP_SOLVER_PBF) {
        vtp::PbfArgs a = pbf_args();
        vtp::pbf_init_boundary(st, a, u.bncnt, u.bnbr, L.ell_stride);
        // boundary volumes live in vol[]; masses in pos.w of both buffers (kernel writes both)
        CU(cudaMemcpyAsync(pos.n() + L.nf, pos.c() + L.nf, (size_t)L.nb * sizeof(float4), cudaMemcpyDeviceToDevice, st));
    } else {
        // v* = v (init_cuda), boundary v* = boundary v.
        for (int k = 0; k < 2; ++k)
            CU(cudaMemcpyAsync(vadv.b[k], vel.c(), (size_t)n * sizeof(float4), cudaMemcpyDeviceToDevice, st));
        vtp::DfsphArgs a = dfsph_args();
        vtp::dfsph_rigid_volume(st, a, u.bncnt, u.bnbr, rest_b);
        CU(cudaMemcpyAsync(pos.n() + L.nf, pos.c() + L.nf, (size_t)L.nb * sizeof(float4), cudaMemcpyDeviceToDevice, st));
        if (type != VTP_SOLVER_DFSPH) {
            if ((rc = immct_init(*this))) return rc;
        }
    }
    CU(cudaGetLastError());
    CU(cudaStreamSynchronize(st));
    initialized = true;
    crashed = false;
    if (cfl > 0.f) vtp::dfsph_cfl_refresh(st, dfsph_args(), d_vmax);
    sim_time = 0.f;
    steps_done = 0;
    out_frames = frames_written = 0;
    graphs_ready = false;
    parity = 0;
#undef AL
    return VTP_OK;
}

// ---------------------------------------------------------------- tick

int vtp_solver::enqueue_solve(cudaStream_t s, int which, bool capture) {
    const vtp::NvtxRange nvtx_range(which == 0 ? "vtp divergence solve" : "vtp density solve");
    vtp::DfsphArgs a = dfsph_args(which);
    vtp::dfsph_solve_begin(s, solve + (size_t)which * scenes.size(), loop + which, nscenes());
    PROF(this, "dfsph_solve_pack", vtp::dfsph_solve_pack(s, a));
    launches_per_tick += 2;
    if (capture && device_loop) {
        cudaStreamCaptureStatus cs;
        cudaGraph_t g;
        const cudaGraphNode_t *deps = nullptr;
        size_t ndeps = 0;
        CU(cudaStreamGetCaptureInfo(s, &cs, nullptr, &g, &deps, &ndeps));
        cudaGraphConditionalHandle hnd;
        CU(cudaGraphConditionalHandleCreate(&hnd, g, 1, cudaGraphCondAssignDefault));
        cudaGraphNodeParams cp = {};
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = hnd;
        cp.conditional.type = cudaGraphCondTypeWhile;
        cp.conditional.size = 1;
        cudaGraphNode_t node;
        CU(cudaGraphAddNode(&node, g, deps, ndeps, &cp));
        cudaGraph_t body = cp.conditional.phGraph_out[0];
        CU(cudaStreamUpdateCaptureDependencies(s, &node, 1, cudaStreamSetCaptureDependencies));
        CU(cudaStreamBeginCaptureToGraph(side, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
        if (scenes.size() == 1) {
            // One scene (every mixture solver, and DFSPH unbatched): the stop test reads only
            // solve_a's residual partials, so it runs as a second branch beside solve_b.  The
            // loop ends when the scene stops, so solve_b (the iteration's last velocity
            // update, as in vfsph_div) runs unconditionally.
            vtp::DfsphArgs sa = type == VTP_SOLVER_DFSPH ? a : immct_solve_args(*this, which);
            vtp::dfsph_solve_a(side, sa, block);
            CU(cudaEventRecord(ev_fork, side));
            CU(cudaStreamWaitEvent(side2, ev_fork, 0));
            vtp::dfsph_solve_end(side2, solve_ctl(which, hnd, 1), partials, d_status);
            sa.state = nullptr;
            vtp::dfsph_solve_b(side, sa, block);
            CU(cudaEventRecord(ev_join, side2));
            CU(cudaStreamWaitEvent(side, ev_join, 0));
        } else {
            // Batched scenes: the same fork; solve_b follows solve_a's record of the tiles it
            // ran this iteration, since the stop test beside it may stop a scene whose tiles
            // this iteration's solve_b must still update.
            vtp::DfsphArgs sa = a;
            sa.tile_ran = d_tile_ran;
            vtp::dfsph_solve_a(side, sa, block);
            CU(cudaEventRecord(ev_fork, side));
            CU(cudaStreamWaitEvent(side2, ev_fork, 0));
            vtp::dfsph_solve_end(side2, solve_ctl(which, hnd, 1), partials, d_status);
            vtp::dfsph_solve_b(side, sa, block);
            CU(cudaEventRecord(ev_join, side2));
            CU(cudaStreamWaitEvent(side, ev_join, 0));
        }
        cudaGraph_t out;
        CU(cudaStreamEndCapture(side, &out));
        return VTP_OK;  // the body's 3 launches per iteration are added from the iteration totals
    }
    // Host-driven loop (reference structure, but only 8 bytes cross PCIe per iteration).
    for (uint32_t it = 0; it < 101; ++it) {
        if (type == VTP_SOLVER_DFSPH) {
            PROF(this, "dfsph_solve_a", vtp::dfsph_solve_a(s, a, block));
            PROF(this, "dfsph_solve_b", vtp::dfsph_solve_b(s, a, block));
        } else {
            immct_solve_ab(*this, s, which);
        }
        PROF(this, "dfsph_solve_end",
             vtp::dfsph_solve_end(s, solve_ctl(which, cudaGraphConditionalHandle{}, 0), partials, d_status));
        launches_per_tick += 3;
        CU(cudaMemcpyAsync(h_pinned + 2, &loop[which].running, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
        CU(cudaStreamSynchronize(s));
        if (!h_pinned[2]) break;
    }
    return VTP_OK;
}

int vtp_solver::enqueue_pbf_substep(cudaStream_t s, const PbfTapeSlot *tape) {
    const vtp::NvtxRange nvtx_range(tape ? "vtp PBF substep (recorded)" : "vtp PBF substep");
    // PBFSolver::tick (PBFSolver.cpp:326-376): external force fused into the sort, neighbour
    // lists, `iterations` constraint passes, XSPH.  With `tape` the lists are built into the
    // tape and the intermediate states are copied out (differentiable mode).
    const size_t nf = L.nf;
    const vtp::PdlScope pdl_scope(pdl);
    vtp::Carry none{};
    vtp::ugns_sort(s, scn(), nbuckets, 0, L.nf, pos.c(), pos.n(), vel.c(), vel.n(), orig.c(), orig.n(), none, dt, u,
                   u.fstart, prof);
    pos.swap(); vel.swap(); orig.swap();
    uint32_t *lnbr = tape ? tape->nbr : u.nbr, *lcnt = tape ? tape->ncnt : u.ncnt;
    PROF(this, "ugns_lists", vtp::ugns_build_lists(s, scn(), L, 0, L.nf, pos.c(), orig.c(), u, lnbr, lcnt,
                                                   d_status, d_overflow, block));
    launches_per_tick += 7;  // hash, 3 scan kernels, scatter, rank/reorder, lists
    if (tape && nf) {
        CU(cudaMemcpyAsync(tape->orig, orig.c(), nf * sizeof(uint32_t), cudaMemcpyDeviceToDevice, s));
        CU(cudaMemcpyAsync(tape->x[0], pos.c(), nf * sizeof(float4), cudaMemcpyDeviceToDevice, s));
    }
    for (int it = 0; it < iterations; ++it) {
        vtp::PbfArgs a = pbf_args();
        a.nbr = lnbr;
        a.ncnt = lcnt;
        if (tape) {
            a.density = tape->rho[it];
            a.lambda = tape->lam[it];
        }
        PROF(this, "pbf_lambda", vtp::pbf_lambda(s, a, block));
        PROF(this, "pbf_dx", vtp::pbf_dx(s, a, block));
        pos.swap();
        launches_per_tick += 2;
        if (tape && nf) CU(cudaMemcpyAsync(tape->x[it + 1], pos.c(), nf * sizeof(float4), cudaMemcpyDeviceToDevice, s));
    }
    if (tape && nf) CU(cudaMemcpyAsync(tape->v, vel.c(), nf * sizeof(float4), cudaMemcpyDeviceToDevice, s));
    vtp::PbfArgs a = pbf_args();
    a.nbr = lnbr;
    a.ncnt = lcnt;
    PROF(this, "pbf_xsph", vtp::pbf_xsph(s, a, block));
    pos.swap(); vel.swap();
    launches_per_tick += 1;
    return VTP_OK;
}

int vtp_solver::enqueue_tick(cudaStream_t s, bool capture) {
    int rc;
    if (type == VTP_SOLVER_PBF) return enqueue_pbf_substep(s, nullptr);
    if (type != VTP_SOLVER_DFSPH) return immct_enqueue_tick(*this, s, capture);
    if (cfl > 0.f) {
        PROF(this, "dfsph_cfl", vtp::dfsph_cfl_step(s, cfl, 2.f * radius, dt, d_vmax, d_cfl, d_cfl + 1));
        launches_per_tick += 1;
    }
    vtp::Carry carry{};
    carry.nf4 = 1;
    carry.src4[0] = vadv.c();
    carry.dst4[0] = vadv.n();
    {
        const vtp::NvtxRange r("vtp neighbour search");
        vtp::ugns_sort(s, scn(), nbuckets, 0, L.nf, pos.c(), pos.n(), vel.c(), vel.n(), orig.c(), orig.n(), carry,
                       0.f, u, u.fstart, prof);
    }
    const vtp::NvtxRange nvtx_lists("vtp neighbour lists and DFSPH passes");
    pos.swap(); vel.swap(); orig.swap(); vadv.swap();
    if (staged) {
        PROF(this, "ugns_lists", vtp::ugns_build_lists_staged(s, scn(), L, stg, pos.c(), u.nbr, u.ncnt, d_status,
                                                              d_overflow));
    } else {
        PROF(this, "ugns_lists", vtp::ugns_build_lists(s, scn(), L, 0, L.nf, pos.c(), orig.c(), u, u.nbr, u.ncnt,
                                                       d_status, d_overflow, block));
    }
    PROF(this, "dfsph_ratio_alpha", vtp::dfsph_ratio_alpha(s, dfsph_args(), block));
    launches_per_tick += 8;  // neighbour search (7) + ratio/alpha
    if ((rc = enqueue_solve(s, 0, capture))) return rc;
    vtp::DfsphArgs a = dfsph_args();
    PROF(this, "dfsph_pressure_pack", vtp::dfsph_pressure_pack(s, a));
    launches_per_tick += 1;
    if (gamma == 0.f) {
        // Tension terms are exactly zero when gamma == 0 (-0 * finite); the normal pass is skipped.
        PROF(this, "dfsph_viscosity", vtp::dfsph_viscosity(s, a, block));
        launches_per_tick += 1;
    } else {
        PROF(this, "dfsph_vis_normal", vtp::dfsph_vis_normal(s, a, block));
        PROF(this, "dfsph_tension", vtp::dfsph_tension(s, a, block));
        launches_per_tick += 2;
    }
    vel.swap(); vadv.swap();
    if ((rc = enqueue_solve(s, 1, capture))) return rc;
    PROF(this, "dfsph_finalize", vtp::dfsph_finalize(s, dfsph_args()));
    launches_per_tick += 1;
    return VTP_OK;
}

int vtp_solver::build_graphs() {
    // Capture two substep graphs: the double buffers swap an odd number of
    // times per substep, so the second graph starts where the first ended.
    int start_state[4] = {pos.cur, vel.cur, orig.cur, vadv.cur};
    for (int p = 0; p < 2; ++p) {
        gstate[p][0] = pos.cur; gstate[p][1] = vel.cur; gstate[p][2] = orig.cur; gstate[p][3] = vadv.cur;
        launches_per_tick = 0;
        CU(cudaStreamBeginCapture(st, cudaStreamCaptureModeRelaxed));
        int rc = enqueue_tick(st, true);
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamEndCapture(st, &g);
        if (rc) {
            if (g) cudaGraphDestroy(g);
            return rc;
        }
        if (e != cudaSuccess) return fail(VTP_ERR_CUDA, std::string("capture: ") + cudaGetErrorString(e));
        e = cudaGraphInstantiate(&gexec[p], g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) return fail(VTP_ERR_CUDA, std::string("instantiate: ") + cudaGetErrorString(e));
    }
    if (imm) immct_set_parity(*this, orig.cur);
    if (pos.cur != start_state[0] || vel.cur != start_state[1] || orig.cur != start_state[2] ||
        vadv.cur != start_state[3])
        return fail(VTP_ERR_STATE, "substep buffer parity does not repeat after two substeps");
    graphs_ready = true;
    parity = 0;
    return VTP_OK;
}

int vtp_solver::sync_parity() {
    // Direct launches (profiling, host loops) may leave the double buffers in
    // either state; pick the graph whose start state matches.
    for (int p = 0; p < 2; ++p) {
        if (pos.cur == gstate[p][0] && vel.cur == gstate[p][1] && orig.cur == gstate[p][2] &&
            vadv.cur == gstate[p][3]) {
            parity = p;
            return VTP_OK;
        }
    }
    return fail(VTP_ERR_STATE, "double-buffer state matches neither substep graph");
}

int vtp_solver::check_status() {
    CU(cudaMemcpyAsync(h_pinned, d_status, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    CU(cudaMemcpyAsync(h_pinned + 1, d_overflow, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    CU(cudaStreamSynchronize(st));
    return apply_status(h_pinned[0], h_pinned[1]);
}

int vtp_solver::apply_status(uint32_t status_bits, uint32_t overflow) {
    stats.status_bits |= status_bits;
    stats.neighbor_overflow = overflow;
    if (status_bits & vtp::ST_NOT_CONVERGED) {
        crashed = true;
        return VTP_NOT_CONVERGED;
    }
    if (status_bits & vtp::ST_NAN) {
        crashed = true;
        return VTP_ERR_NAN;
    }
    return VTP_OK;
}

int vtp_solver::tick_n(uint32_t n, const std::function<int()> &tail) {
    const vtp::NvtxRange nvtx_range("vtp tick");
    int rc;
    if (!initialized && (rc = initialize())) return rc;
    if (crashed) return fail(VTP_NOT_CONVERGED, std::string(solver_key(type)) + "Solver is crashed.");
    const bool solves = type != VTP_SOLVER_PBF;
    if (solves) {
        CU(cudaMemsetAsync(solve, 0, 2 * scenes.size() * sizeof(vtp::SolveState), st));
        CU(cudaMemsetAsync(loop, 0, 2 * sizeof(vtp::LoopState), st));
    }
    if (use_graphs && !graphs_ready) {
        if ((rc = build_graphs())) {
            // A failed capture leaves the stream usable; fall back to direct launches.
            cudaGetLastError();
            use_graphs = false;
            g_last_error.clear();
        }
    }
    if (use_graphs && (rc = sync_parity())) return rc;
    CU(cudaMemsetAsync(d_overflow, 0, sizeof(uint32_t), st));
    CU(cudaEventRecord(ev[0], st));
    uint64_t launches = 0;
    for (uint32_t k = 0; k < n; ++k) {
        if (use_graphs) {
            CU(cudaGraphLaunch(gexec[parity], st));
            int np = parity ^ 1;
            pos.cur = gstate[np][0]; vel.cur = gstate[np][1]; orig.cur = gstate[np][2]; vadv.cur = gstate[np][3];
            if (imm) immct_set_parity(*this, orig.cur);
            parity = np;
        } else {
            launches_per_tick = 0;
            if ((rc = enqueue_tick(st, false))) return rc;
            launches += launches_per_tick;
        }
        if (cfl > 0.f) {
            // adaptive step: the simulated time lives on the device; read it when an export needs it
            if (export_enabled) {
                CU(cudaMemcpyAsync(h_pinned + 6, d_cfl + 1, sizeof(float), cudaMemcpyDeviceToHost, st));
                CU(cudaStreamSynchronize(st));
                std::memcpy(&sim_time, h_pinned + 6, sizeof(float));
            }
        } else {
            sim_time += dt;
        }
        ++steps_done;
        if ((rc = maybe_export())) return rc;
        if (solves && stop_on_crash && k + 1 < n) {
            // The reference stops ticking after a solve ran past 100 iterations (the last
            // substep's status comes back with the end-of-tick readback below).
            if ((rc = check_status())) {
                stats.steps_done = steps_done;
                return fail(rc, std::string(solver_key(type)) + ": pressure solve exceeded 100 iterations");
            }
        }
    }
    CU(cudaEventRecord(ev[2], st));
    if (tail && (rc = tail())) return rc;
    // What the host reports after the tick comes back in one readback behind one
    // synchronisation: the status words, the adaptive step, the solve and loop states.
    const size_t S = scenes.size();
    const size_t off_solve = 16, off_loop = off_solve + 2 * S * sizeof(vtp::SolveState);
    const size_t need = off_loop + 2 * sizeof(vtp::LoopState);
    if (need > h_tick_bytes) {
        if (h_tick) cudaFreeHost(h_tick), h_tick = nullptr, h_tick_bytes = 0;
        CU(cudaMallocHost((void **)&h_tick, need));
        h_tick_bytes = need;
    }
    uint32_t *hw = reinterpret_cast<uint32_t *>(h_tick);
    const vtp::SolveState *hs = reinterpret_cast<const vtp::SolveState *>(h_tick + off_solve);
    const vtp::LoopState *hl = reinterpret_cast<const vtp::LoopState *>(h_tick + off_loop);
    CU(cudaMemcpyAsync(hw, d_status, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    CU(cudaMemcpyAsync(hw + 1, d_overflow, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    if (cfl > 0.f) CU(cudaMemcpyAsync(hw + 2, d_cfl, 2 * sizeof(float), cudaMemcpyDeviceToHost, st));
    if (solves) {
        CU(cudaMemcpyAsync(h_tick + off_solve, solve, 2 * S * sizeof(vtp::SolveState), cudaMemcpyDeviceToHost, st));
        CU(cudaMemcpyAsync(h_tick + off_loop, loop, 2 * sizeof(vtp::LoopState), cudaMemcpyDeviceToHost, st));
    }
    CU(cudaStreamSynchronize(st));
    CU(cudaGetLastError());
    CU(cudaEventElapsedTime(&stage_ms[2], ev[0], ev[2]));
    if (cfl > 0.f) {
        float dev[2];
        std::memcpy(dev, hw + 2, sizeof(dev));
        last_dt = dev[0];
        sim_time = dev[1];
    }
    if ((rc = apply_status(hw[0], hw[1]))) {
        if (solves && stop_on_crash) {
            stats.steps_done = steps_done;
            return fail(rc, std::string(solver_key(type)) + ": pressure solve exceeded 100 iterations");
        }
        return fail(rc, "solver status after tick");
    }
    if (solves) {
        fill_solve_stats(hs);
        stats = scene_stats[0];
        // per solve-loop iteration: solve_a, solve_b, solve_end
        if (use_graphs) launches = (uint64_t)n * launches_per_tick + 3 * (hl[0].total + hl[1].total);
    } else if (use_graphs) {
        launches = (uint64_t)n * launches_per_tick;
    }
    if (imm) {
        uint64_t body = 0;
        stats.phase_retries = immct_last_retries(*this, &body);
        if (use_graphs) launches += body;   // launched inside the retry loop's WHILE node
    }
    last_launches = launches;
    stats.steps_done = steps_done;
    stats.sim_time = sim_time;
    stats.last_dt = cfl > 0.f ? last_dt : dt;
    return VTP_OK;
}

void vtp_solver::fill_solve_stats(const vtp::SolveState *hs) {
    const size_t S = scenes.size();
    scene_stats.assign(S, stats);
    for (size_t k = 0; k < S; ++k) {
        vtp_stats &o = scene_stats[k];
        o.last_div_iters = hs[k].last_iters;
        o.last_incomp_iters = hs[S + k].last_iters;
        o.total_div_iters = hs[k].total_iters;
        o.total_incomp_iters = hs[S + k].total_iters;
        o.last_div_residual = hs[k].residual;
        o.last_incomp_residual = hs[S + k].residual;
    }
}

// ---------------------------------------------------------------- fields

static size_t field_elems(const vtp_solver &s, int f) {
    switch (f) {
        case VTP_FIELD_POS: case VTP_FIELD_VEL: case VTP_FIELD_COLOR: return 3;
        case VTP_FIELD_MAT: case VTP_FIELD_MASS: case VTP_FIELD_VOLUME: case VTP_FIELD_DENSITY:
        case VTP_FIELD_LAMBDA: case VTP_FIELD_ALPHA: case VTP_FIELD_KAPPA: case VTP_FIELD_REST_DENSITY:
        case VTP_FIELD_DELTA: return 1;
        case VTP_FIELD_CD: return s.imm ? 1 : 0;
        case VTP_FIELD_VOL_FRAC: return s.imm ? immct_phase_count(s) : 0;
        case VTP_FIELD_PHASE_VEL: return s.imm ? 3 * immct_phase_count(s) : 0;
        case VTP_FIELD_CONFORMATION: case VTP_FIELD_STRESS: return s.imm ? 9 : 0;
    }
    return 0;
}

int vtp_solver::get_field(int f, void *host, size_t bytes) {
    if (!initialized) return fail(VTP_ERR_STATE, "get_field before initialize");
    const size_t ne = field_elems(*this, f);
    if (ne == 0) return fail(VTP_ERR_ARG, "field not available for this solver");
    if (!host || bytes != (size_t)L.n * ne * 4) return fail(VTP_ERR_ARG, "wrong byte count for field");
    const uint32_t n = L.n;
    if (f == VTP_FIELD_COLOR) {
        if (imm) {
            // color = sum_k alpha_k phaseRestColor_k (update_color_cuda, IMMCTCudaImpl.cu:512-524)
            const int P = immct_phase_count(*this);
            std::vector<float> fr((size_t)L.n * P);
            int rc = get_field(VTP_FIELD_VOL_FRAC, fr.data(), fr.size() * 4);
            if (rc) return rc;
            immct_color(*this, fr.data(), (float *)host);
            return VTP_OK;
        }
        memcpy(host, hcolor.data(), bytes);
        return VTP_OK;
    }
    if (imm && (f == VTP_FIELD_MASS || f == VTP_FIELD_REST_DENSITY || f == VTP_FIELD_CD ||
                f == VTP_FIELD_VOL_FRAC || f == VTP_FIELD_PHASE_VEL || f == VTP_FIELD_CONFORMATION ||
                f == VTP_FIELD_STRESS)) {
        int rc = ensure_stage(bytes);
        if (rc) return rc;
        if ((rc = immct_get_field(*this, f, stage, ne))) return rc;
        cudaError_t e = cudaMemcpy(host, stage, bytes, cudaMemcpyDeviceToHost);
        return e == cudaSuccess ? VTP_OK : fail(VTP_ERR_CUDA, cudaGetErrorString(e));
    }
    if (f == VTP_FIELD_MAT) { memcpy(host, hmat.data(), bytes); return VTP_OK; }
    int rc = ensure_stage(bytes);
    if (rc) return rc;
    float *tmp = stage;
    auto fluid_scalar = [&](const float *src, float boundary_value) -> int {
        // fluid rows from src, boundary rows constant
        std::vector<float> hv(n, boundary_value);
        std::vector<uint32_t> ids(n);
        if (L.nf) {
            std::vector<float> fv(L.nf);
            if (cudaMemcpy(fv.data(), src, L.nf * sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess) return 1;
            if (cudaMemcpy(ids.data(), orig.c(), n * sizeof(uint32_t), cudaMemcpyDeviceToHost) != cudaSuccess) return 1;
            for (uint32_t r = 0; r < L.nf; ++r) hv[ids[r]] = fv[r];
        }
        memcpy(host, hv.data(), bytes);
        return 0;
    };
    switch (f) {
        case VTP_FIELD_POS: vtp::scatter_f4_to_orig(st, n, pos.c(), orig.c(), tmp); break;
        case VTP_FIELD_VEL: vtp::scatter_f4_to_orig(st, n, vel.c(), orig.c(), tmp); break;
        case VTP_FIELD_MASS:
        case VTP_FIELD_VOLUME:
        case VTP_FIELD_REST_DENSITY: {
            std::vector<float4> p4(n);
            std::vector<uint32_t> ids(n);
            std::vector<float> vv;
            CU(cudaMemcpy(p4.data(), pos.c(), n * sizeof(float4), cudaMemcpyDeviceToHost));
            CU(cudaMemcpy(ids.data(), orig.c(), n * sizeof(uint32_t), cudaMemcpyDeviceToHost));
            std::vector<float> rb(L.nb);
            if (type != VTP_SOLVER_PBF && L.nb) CU(cudaMemcpy(rb.data(), rest_b, L.nb * sizeof(float), cudaMemcpyDeviceToHost));
            if (type == VTP_SOLVER_PBF) {
                vv.resize(n);
                CU(cudaMemcpy(vv.data(), vol, n * sizeof(float), cudaMemcpyDeviceToHost));
            }
            std::vector<float> out(n);
            for (uint32_t r = 0; r < n; ++r) {
                float v = 0.f;
                bool fl = r < L.nf;
                if (type == VTP_SOLVER_PBF) {
                    if (f == VTP_FIELD_MASS) v = p4[r].w;
                    else if (f == VTP_FIELD_VOLUME) v = vv[r];
                    else v = fl ? rho_f : rho_b;
                } else if (type == VTP_SOLVER_DFSPH) {
                    if (f == VTP_FIELD_VOLUME) v = p4[r].w;
                    else if (f == VTP_FIELD_MASS) v = fl ? rho_f * vol0 : 0.f;
                    else v = fl ? rho_f : rb[r - L.nf];
                } else {
                    v = p4[r].w;   // IMM / IMM-CT volume (mass and rest density handled above)
                }
                out[ids[r]] = v;
            }
            memcpy(host, out.data(), bytes);
            return VTP_OK;
        }
        case VTP_FIELD_DENSITY:
            rc = fluid_scalar(type == VTP_SOLVER_PBF ? density : ratio, 0.f);
            return rc ? fail(VTP_ERR_CUDA, "field copy failed") : VTP_OK;
        case VTP_FIELD_LAMBDA:
            if (type != VTP_SOLVER_PBF) return fail(VTP_ERR_ARG, "lambda is a PBF field");
            rc = fluid_scalar(lambda, 0.f);
            return rc ? fail(VTP_ERR_CUDA, "field copy failed") : VTP_OK;
        case VTP_FIELD_ALPHA:
        case VTP_FIELD_KAPPA:
        case VTP_FIELD_DELTA:
            if (type == VTP_SOLVER_PBF) return fail(VTP_ERR_ARG, "not a PBF field");
            rc = fluid_scalar(f == VTP_FIELD_ALPHA ? alpha : f == VTP_FIELD_KAPPA ? kappa : delta, 0.f);
            return rc ? fail(VTP_ERR_CUDA, "field copy failed") : VTP_OK;
        default:
            rc = immct_get_field(*this, f, tmp, ne);
            if (rc) return rc;
            break;
    }
    cudaError_t e = cudaMemcpyAsync(host, tmp, bytes, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return fail(VTP_ERR_CUDA, cudaGetErrorString(e));
    return VTP_OK;
}

int vtp_solver::set_field(int f, const void *host, size_t bytes) {
    if (!initialized) return fail(VTP_ERR_STATE, "set_field before initialize");
    if (f != VTP_FIELD_POS && f != VTP_FIELD_VEL) return fail(VTP_ERR_ARG, "only pos / vel can be set");
    if (!host || bytes != (size_t)L.n * 12) return fail(VTP_ERR_ARG, "wrong byte count for field");
    int rc = ensure_stage(bytes);
    if (rc) return rc;
    float *tmp = stage;
    cudaError_t e = cudaMemcpyAsync(tmp, host, bytes, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) {
        // Only fluid rows move; boundary rows are static and stay as sorted at initialize.
        DB<float4> &d = f == VTP_FIELD_POS ? pos : vel;
        vtp::gather_orig_to_f4(st, L.nf, tmp, orig.c(), d.c(), 1);
        if (f == VTP_FIELD_VEL && vadv.c()) vtp::gather_orig_to_f4(st, L.nf, tmp, orig.c(), vadv.c(), 1);
        if (f == VTP_FIELD_VEL && cfl > 0.f) vtp::dfsph_cfl_refresh(st, dfsph_args(), d_vmax);
        e = cudaStreamSynchronize(st);
    }
    if (e != cudaSuccess) return fail(VTP_ERR_CUDA, cudaGetErrorString(e));
    return VTP_OK;
}

// ---------------------------------------------------------------- C ABI

extern "C" {

const char *vtp_status_string(int s) {
    switch (s) {
        case VTP_OK: return "ok";
        case VTP_ERR_CONFIG: return "invalid config";
        case VTP_ERR_CUDA: return "CUDA error";
        case VTP_NOT_CONVERGED: return "pressure solve did not converge within 100 iterations";
        case VTP_ERR_NAN: return "non-finite state";
        case VTP_ERR_TIMEOUT: return "device wait timed out";
        case VTP_ERR_BOUNDS: return "size or index out of bounds";
        case VTP_ERR_STATE: return "call out of order";
        case VTP_ERR_ARG: return "invalid argument";
        case VTP_ERR_NOMEM: return "out of device memory";
    }
    return "unknown status";
}

const char *vtp_version(void) { return "vtp 0.1 sm_100a"; }

const char *vtp_last_error(void) { return g_last_error.c_str(); }

int vtp_solver_create(int solver_type, vtp_solver **out) {
    if (!out) return fail(VTP_ERR_ARG, "null out");
    *out = nullptr;
    if (solver_type < VTP_SOLVER_PBF || solver_type > VTP_SOLVER_IMMCT)
        return fail(VTP_ERR_ARG, "unknown solver type");
    auto *s = new (std::nothrow) vtp_solver();
    if (!s) return fail(VTP_ERR_NOMEM, "host allocation failed");
    s->type = solver_type;
    s->cfg = default_config(solver_type);
    *out = s;
    return VTP_OK;
}

int vtp_solver_set_config(vtp_solver *s, const char *json_text) {
    if (!s || !json_text) return fail(VTP_ERR_ARG, "null argument");
    json c;
    try {
        c = json::parse(json_text);
    } catch (const std::exception &e) {
        return fail(VTP_ERR_CONFIG, std::string("JSON parse error: ") + e.what());
    }
    if (s->initialized) return fail(VTP_ERR_STATE, "setConfig after initialize");
    return s->parse_config(c);
}

int vtp_solver_attach_object(vtp_solver *s, const float *pos, uint32_t n, const float *vel, const char *object_json) {
    if (!s || !object_json) return fail(VTP_ERR_ARG, "null argument");
    json o;
    try {
        o = json::parse(object_json);
    } catch (const std::exception &e) {
        return fail(VTP_ERR_CONFIG, std::string("JSON parse error: ") + e.what());
    }
    try {
        return s->attach(pos, n, vel, o);
    } catch (const std::exception &e) {
        return fail(VTP_ERR_CONFIG, std::string("object config error: ") + e.what());
    }
}

int vtp_solver_add_scene(vtp_solver *s, const char *json_text, uint32_t *scene_index) {
    if (!s || !json_text) return fail(VTP_ERR_ARG, "null argument");
    json c;
    try {
        c = json::parse(json_text);
    } catch (const std::exception &e) {
        return fail(VTP_ERR_CONFIG, std::string("JSON parse error: ") + e.what());
    }
    return s->add_scene(c, scene_index);
}

int vtp_solver_get_scene_stats(vtp_solver *s, uint32_t scene, vtp_stats *out) {
    if (!s || !out) return fail(VTP_ERR_ARG, "null argument");
    if (scene >= s->scenes.size()) return fail(VTP_ERR_ARG, "scene index out of range");
    *out = s->stats;
    if (scene < s->scene_stats.size()) {
        const vtp_stats &k = s->scene_stats[scene];
        out->last_div_iters = k.last_div_iters;
        out->last_incomp_iters = k.last_incomp_iters;
        out->total_div_iters = k.total_div_iters;
        out->total_incomp_iters = k.total_incomp_iters;
        out->last_div_residual = k.last_div_residual;
        out->last_incomp_residual = k.last_incomp_residual;
    }
    return VTP_OK;
}

int vtp_solver_initialize(vtp_solver *s) {
    if (!s) return fail(VTP_ERR_ARG, "null solver");
    try {
        int rc = s->initialize();
        if (rc) s->release();
        return rc;
    } catch (const std::exception &e) {
        s->release();
        return fail(VTP_ERR_CONFIG, e.what());
    }
}

int vtp_solver_tick_n_steps(vtp_solver *s, uint32_t n) {
    if (!s) return fail(VTP_ERR_ARG, "null solver");
    return s->tick_n(n);
}

int vtp_solver_run(vtp_solver *s) {
    if (!s) return fail(VTP_ERR_ARG, "null solver");
    int rc;
    if (!s->initialized && (rc = s->initialize())) return rc;
    // while (cur_simTime < animationTime) tick()   (PBFSolver.cpp:134-143)
    while (s->sim_time < s->anim_time) {
        if ((rc = s->tick_n(1))) return rc;
    }
    return VTP_OK;
}

int vtp_solver_reset(vtp_solver *s) {
    if (!s) return fail(VTP_ERR_ARG, "null solver");
    s->cfg = default_config(s->type);
    return VTP_OK;
}

void vtp_solver_destroy(vtp_solver *s) { delete s; }

int vtp_solver_get_config(vtp_solver *s, char *buf, size_t buf_bytes, size_t *needed) {
    if (!s) return fail(VTP_ERR_ARG, "null solver");
    std::string t = s->cfg.dump();
    if (needed) *needed = t.size() + 1;
    if (!buf) return VTP_OK;
    if (buf_bytes < t.size() + 1) return fail(VTP_ERR_ARG, "buffer too small");
    memcpy(buf, t.c_str(), t.size() + 1);
    return VTP_OK;
}

int vtp_solver_get_stats(vtp_solver *s, vtp_stats *out) {
    if (!s || !out) return fail(VTP_ERR_ARG, "null argument");
    *out = s->stats;
    return VTP_OK;
}

int vtp_solver_particle_counts(vtp_solver *s, uint32_t *n_total, uint32_t *n_fluid, uint32_t *n_boundary,
                               uint32_t *n_phases) {
    if (!s) return fail(VTP_ERR_ARG, "null solver");
    uint32_t n = (uint32_t)(s->hpos.size() / 3), nf = 0;
    for (auto &o : s->objs)
        if (o.mat == 0) nf += o.end - o.start;
    if (n_total) *n_total = n;
    if (n_fluid) *n_fluid = nf;
    if (n_boundary) *n_boundary = n - nf;
    if (n_phases) *n_phases = s->imm ? (uint32_t)immct_phase_count(*s) : 0;
    return VTP_OK;
}

int vtp_solver_get_field(vtp_solver *s, int field, void *host, size_t bytes) {
    if (!s) return fail(VTP_ERR_ARG, "null solver");
    return s->get_field(field, host, bytes);
}

int vtp_solver_set_field(vtp_solver *s, int field, const void *host, size_t bytes) {
    if (!s) return fail(VTP_ERR_ARG, "null solver");
    return s->set_field(field, host, bytes);
}

int vtp_solver_get_field_range(vtp_solver *s, int field, uint32_t first, uint32_t count, void *host, size_t bytes) {
    if (!s || (!host && count)) return fail(VTP_ERR_ARG, "null argument");
    if (!s->initialized) return fail(VTP_ERR_STATE, "get_field before initialize");
    if ((uint64_t)first + count > s->L.n) return fail(VTP_ERR_ARG, "particle range out of bounds");
    if (field != VTP_FIELD_POS && field != VTP_FIELD_VEL) {
        // other fields: through the full-size path
        const size_t ne = bytes / (count ? count : 1) / 4;
        std::vector<float> all((size_t)s->L.n * ne);
        int rc = s->get_field(field, all.data(), all.size() * 4);
        if (rc) return rc;
        if (bytes != (size_t)count * ne * 4) return fail(VTP_ERR_ARG, "wrong byte count for field");
        memcpy(host, all.data() + (size_t)first * ne, bytes);
        return VTP_OK;
    }
    if (bytes != (size_t)count * 12) return fail(VTP_ERR_ARG, "wrong byte count for field");
    if (!count) return VTP_OK;
    int rc = s->ensure_stage(bytes);
    if (rc) return rc;
    const DB<float4> &d = field == VTP_FIELD_POS ? s->pos : s->vel;
    vtp::scatter_f4_range(s->st, s->L.n, d.c(), s->orig.c(), first, count, s->stage);
    cudaError_t e = cudaMemcpyAsync(host, s->stage, bytes, cudaMemcpyDeviceToHost, s->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->st);
    return e == cudaSuccess ? VTP_OK : fail(VTP_ERR_CUDA, cudaGetErrorString(e));
}

int vtp_solver_set_field_range(vtp_solver *s, int field, uint32_t first, uint32_t count, const void *host,
                               size_t bytes) {
    if (!s || (!host && count)) return fail(VTP_ERR_ARG, "null argument");
    if (!s->initialized) return fail(VTP_ERR_STATE, "set_field before initialize");
    if (field != VTP_FIELD_POS && field != VTP_FIELD_VEL) return fail(VTP_ERR_ARG, "only pos / vel can be set");
    if ((uint64_t)first + count > s->L.n) return fail(VTP_ERR_ARG, "particle range out of bounds");
    if (bytes != (size_t)count * 12) return fail(VTP_ERR_ARG, "wrong byte count for field");
    if (!count) return VTP_OK;
    int rc = s->ensure_stage(bytes);
    if (rc) return rc;
    cudaError_t e = cudaMemcpyAsync(s->stage, host, bytes, cudaMemcpyHostToDevice, s->st);
    if (e == cudaSuccess) {
        // Only fluid rows move; boundary rows are static and stay as sorted at initialize.
        DB<float4> &d = field == VTP_FIELD_POS ? s->pos : s->vel;
        float4 *also = field == VTP_FIELD_VEL && s->vadv.c() ? s->vadv.c() : nullptr;
        vtp::gather_f4_range(s->st, s->L.nf, s->stage, s->orig.c(), first, count, d.c(), also);
        if (field == VTP_FIELD_VEL && s->cfl > 0.f) vtp::dfsph_cfl_refresh(s->st, s->dfsph_args(), s->d_vmax);
        e = cudaStreamSynchronize(s->st);
    }
    return e == cudaSuccess ? VTP_OK : fail(VTP_ERR_CUDA, cudaGetErrorString(e));
}

int vtp_host_alloc(size_t bytes, void **ptr) {
    if (!ptr) return fail(VTP_ERR_ARG, "null argument");
    *ptr = nullptr;
    cudaError_t e = cudaHostAlloc(ptr, bytes ? bytes : 1, cudaHostAllocDefault);
    if (e != cudaSuccess) return fail(VTP_ERR_NOMEM, std::string("cudaHostAlloc: ") + cudaGetErrorString(e));
    return VTP_OK;
}

void vtp_host_free(void *ptr) {
    if (ptr) cudaFreeHost(ptr);
}

int vtp_selftest_cube(uint32_t *mismatches, uint32_t *max_ulp) {
    if (!mismatches || !max_ulp) return fail(VTP_ERR_ARG, "null argument");
    cudaStream_t st;
    cudaError_t e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
    if (e != cudaSuccess) return fail(VTP_ERR_CUDA, cudaGetErrorString(e));
    const int rc = vtp::selftest_cube(st, mismatches, max_ulp);
    cudaStreamDestroy(st);
    return rc ? fail(VTP_ERR_CUDA, "cube self-test failed to run") : VTP_OK;
}

int vtp_solver_get_state_range(vtp_solver *s, uint32_t first, uint32_t count, float *pos, float *vel) {
    if (!s || ((!pos || !vel) && count)) return fail(VTP_ERR_ARG, "null argument");
    if (!s->initialized) return fail(VTP_ERR_STATE, "get_state before initialize");
    if ((uint64_t)first + count > s->L.n) return fail(VTP_ERR_ARG, "particle range out of bounds");
    if (!count) return VTP_OK;
    const size_t b = (size_t)count * 12;
    int rc = s->ensure_stage(2 * b);
    if (rc) return rc;
    float *p3 = s->stage, *v3 = s->stage + (size_t)count * 3;
    vtp::scatter_state_range(s->st, s->L.n, s->pos.c(), s->vel.c(), s->orig.c(), first, count, p3, v3);
    cudaError_t e = cudaMemcpyAsync(pos, p3, b, cudaMemcpyDeviceToHost, s->st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(vel, v3, b, cudaMemcpyDeviceToHost, s->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->st);
    return e == cudaSuccess ? VTP_OK : fail(VTP_ERR_CUDA, cudaGetErrorString(e));
}

int vtp_solver_set_state_range(vtp_solver *s, uint32_t first, uint32_t count, const float *pos, const float *vel) {
    if (!s || ((!pos || !vel) && count)) return fail(VTP_ERR_ARG, "null argument");
    if (!s->initialized) return fail(VTP_ERR_STATE, "set_state before initialize");
    if ((uint64_t)first + count > s->L.n) return fail(VTP_ERR_ARG, "particle range out of bounds");
    if (!count) return VTP_OK;
    const size_t b = (size_t)count * 12;
    int rc = s->ensure_stage(2 * b);
    if (rc) return rc;
    float *p3 = s->stage, *v3 = s->stage + (size_t)count * 3;
    cudaError_t e = cudaMemcpyAsync(p3, pos, b, cudaMemcpyHostToDevice, s->st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(v3, vel, b, cudaMemcpyHostToDevice, s->st);
    if (e == cudaSuccess) {
        // Only fluid rows move; boundary rows are static and stay as sorted at initialize.
        vtp::gather_state_range(s->st, s->L.nf, p3, v3, s->orig.c(), first, count, s->pos.c(), s->vel.c(),
                                s->vadv.c());
        if (s->cfl > 0.f) vtp::dfsph_cfl_refresh(s->st, s->dfsph_args(), s->d_vmax);
        e = cudaStreamSynchronize(s->st);
    }
    return e == cudaSuccess ? VTP_OK : fail(VTP_ERR_CUDA, cudaGetErrorString(e));
}

int vtp_solver_step_state_ranges(vtp_solver *s, uint32_t nranges, const uint32_t *firsts, const uint32_t *counts,
                                 const float *pos_in, const float *vel_in, uint32_t n_steps, float *pos_out,
                                 float *vel_out) {
    if (!s || (nranges && (!firsts || !counts))) return fail(VTP_ERR_ARG, "null argument");
    if (!s->initialized) return fail(VTP_ERR_STATE, "step_state before initialize");
    uint64_t total = 0;
    for (uint32_t k = 0; k < nranges; ++k) {
        if ((uint64_t)firsts[k] + counts[k] > s->L.n) return fail(VTP_ERR_ARG, "particle range out of bounds");
        if (k && firsts[k] < (uint64_t)firsts[k - 1] + counts[k - 1])
            return fail(VTP_ERR_ARG, "particle ranges must be ascending and disjoint");
        total += counts[k];
    }
    if (!total) return s->tick_n(n_steps);
    if (!pos_in || !vel_in || !pos_out || !vel_out) return fail(VTP_ERR_ARG, "null argument");
    const size_t b = (size_t)total * 12;
    int rc = s->ensure_stage(2 * b);
    if (rc) return rc;
    float *p3 = s->stage, *v3 = s->stage + (size_t)total * 3;
    // One range goes by value; several through a {first, count, first slot} table on the device.
    const bool one = nranges == 1;
    if (!one) {
        std::vector<uint32_t> tab(3 * (size_t)nranges);
        uint32_t slot = 0;
        for (uint32_t k = 0; k < nranges; ++k) {
            tab[3 * (size_t)k] = firsts[k];
            tab[3 * (size_t)k + 1] = counts[k];
            tab[3 * (size_t)k + 2] = slot;
            slot += counts[k];
        }
        if ((rc = s->ensure_ranges(nranges))) return rc;
        // from pageable memory: the table is copied out before the call returns
        CU(cudaMemcpyAsync(s->d_ranges, tab.data(), tab.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, s->st));
    }
    // set_state_range's copies and row gather, the substeps, get_state_range's row scatter and
    // copies, all in stream order; the tick's end-of-tick readback synchronises once for all.
    CU(cudaMemcpyAsync(p3, pos_in, b, cudaMemcpyHostToDevice, s->st));
    CU(cudaMemcpyAsync(v3, vel_in, b, cudaMemcpyHostToDevice, s->st));
    if (one)
        vtp::gather_state_range(s->st, s->L.nf, p3, v3, s->orig.c(), firsts[0], counts[0], s->pos.c(), s->vel.c(),
                                s->vadv.c());
    else
        vtp::gather_state_ranges(s->st, s->L.nf, p3, v3, s->orig.c(), s->d_ranges, nranges, s->pos.c(), s->vel.c(),
                                 s->vadv.c());
    if (s->cfl > 0.f) vtp::dfsph_cfl_refresh(s->st, s->dfsph_args(), s->d_vmax);
    CU(cudaGetLastError());
    const uint32_t first0 = firsts[0], count0 = counts[0];
    rc = s->tick_n(n_steps, [&]() -> int {
        if (one)
            vtp::scatter_state_range(s->st, s->L.n, s->pos.c(), s->vel.c(), s->orig.c(), first0, count0, p3, v3);
        else
            vtp::scatter_state_ranges(s->st, s->L.n, s->pos.c(), s->vel.c(), s->orig.c(), s->d_ranges, nranges, p3,
                                      v3);
        CU(cudaMemcpyAsync(pos_out, p3, b, cudaMemcpyDeviceToHost, s->st));
        CU(cudaMemcpyAsync(vel_out, v3, b, cudaMemcpyDeviceToHost, s->st));
        return VTP_OK;
    });
    // On an error the ticks may have returned before their readback: wait for the queued
    // copies, so that the input buffers are read (and the outputs no longer written) on return.
    if (rc) cudaStreamSynchronize(s->st);
    return rc;
}

int vtp_solver_step_state_range(vtp_solver *s, uint32_t first, uint32_t count, const float *pos_in,
                                const float *vel_in, uint32_t n_steps, float *pos_out, float *vel_out) {
    return vtp_solver_step_state_ranges(s, 1, &first, &count, pos_in, vel_in, n_steps, pos_out, vel_out);
}

int vtp_solver_get_neighbors(vtp_solver *s, uint32_t *counts, uint32_t *nbrs, uint32_t max_nbr) {
    if (!s || !counts || !nbrs) return fail(VTP_ERR_ARG, "null argument");
    if (!s->initialized) return fail(VTP_ERR_STATE, "get_neighbors before initialize");
    if (max_nbr != s->maxnbr) return fail(VTP_ERR_ARG, "max_nbr must equal maxNeighborNum");
    const uint32_t n = s->L.n;
    // Neighbour search of the current state, all rows (UniformGirdNeighborSearcher::update on the
    // current positions): re-sort the fluid rows and rebuild both row ranges' lists.  Every
    // substep starts with the same search, so the solver state is unaffected.
    vtp::Carry carry{};
    if (s->vadv.c()) {
        carry.nf4 = 1;
        carry.src4[0] = s->vadv.c();
        carry.dst4[0] = s->vadv.n();
    }
    if (s->imm) immct_fill_carry(*s, carry);
    vtp::ugns_sort(s->st, s->scn(), s->nbuckets, 0, s->L.nf, s->pos.c(), s->pos.n(), s->vel.c(), s->vel.n(),
                   s->orig.c(), s->orig.n(), carry, 0.f, s->u, s->u.fstart);
    // Copy the re-sorted fluid rows back so the buffer parity the substep graphs expect is kept.
    const size_t nf = s->L.nf;
    CU(cudaMemcpyAsync(s->pos.c(), s->pos.n(), nf * sizeof(float4), cudaMemcpyDeviceToDevice, s->st));
    CU(cudaMemcpyAsync(s->vel.c(), s->vel.n(), nf * sizeof(float4), cudaMemcpyDeviceToDevice, s->st));
    CU(cudaMemcpyAsync(s->orig.c(), s->orig.n(), nf * sizeof(uint32_t), cudaMemcpyDeviceToDevice, s->st));
    if (s->vadv.c())
        CU(cudaMemcpyAsync(s->vadv.c(), s->vadv.n(), nf * sizeof(float4), cudaMemcpyDeviceToDevice, s->st));
    if (s->imm) {
        int rc = immct_copy_back(*s);
        if (rc) return rc;
    }
    vtp::ugns_build_lists(s->st, s->scn(), s->L, 0, s->L.nf, s->pos.c(), s->orig.c(), s->u, s->u.nbr, s->u.ncnt,
                          s->d_status, s->d_overflow, s->block);
    vtp::ugns_build_lists(s->st, s->scn(), s->L, s->L.nf, s->L.nb, s->pos.c(), s->orig.c(), s->u, s->u.bnbr,
                          s->u.bncnt, s->d_status, s->d_overflow, s->block);
    uint32_t *dc = nullptr, *dn = nullptr;
    CU(cudaMalloc(&dc, (size_t)n * 4));
    cudaError_t e = cudaMalloc(&dn, (size_t)n * max_nbr * 4);
    if (e != cudaSuccess) { cudaFree(dc); return fail(VTP_ERR_NOMEM, "neighbour export buffer"); }
    vtp::export_neighbors(s->st, s->L, 0, s->L.nf, s->u.nbr, s->u.ncnt, s->orig.c(), max_nbr, dc, dn);
    vtp::export_neighbors(s->st, s->L, s->L.nf, s->L.nb, s->u.bnbr, s->u.bncnt, s->orig.c(), max_nbr, dc, dn);
    e = cudaMemcpyAsync(counts, dc, (size_t)n * 4, cudaMemcpyDeviceToHost, s->st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(nbrs, dn, (size_t)n * max_nbr * 4, cudaMemcpyDeviceToHost, s->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->st);
    cudaFree(dc);
    cudaFree(dn);
    if (e != cudaSuccess) return fail(VTP_ERR_CUDA, cudaGetErrorString(e));
    return VTP_OK;
}

int vtp_solver_get_sorted_order(vtp_solver *s, uint32_t *sorted_ids, uint32_t *cell_ids) {
    if (!s || !sorted_ids || !cell_ids) return fail(VTP_ERR_ARG, "null argument");
    if (!s->initialized) return fail(VTP_ERR_STATE, "get_sorted_order before initialize");
    const uint32_t n = s->L.n;
    uint32_t *di = nullptr, *dk = nullptr;
    CU(cudaMalloc(&di, (size_t)n * 4));
    cudaError_t e = cudaMalloc(&dk, (size_t)n * 4);
    if (e != cudaSuccess) { cudaFree(di); return fail(VTP_ERR_NOMEM, "sorted export buffer"); }
    vtp::export_sorted(s->st, s->scn(), n, s->pos.c(), s->orig.c(), di, dk);
    std::vector<uint32_t> ids(n), keys(n);
    e = cudaMemcpyAsync(ids.data(), di, (size_t)n * 4, cudaMemcpyDeviceToHost, s->st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(keys.data(), dk, (size_t)n * 4, cudaMemcpyDeviceToHost, s->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->st);
    cudaFree(di);
    cudaFree(dk);
    if (e != cudaSuccess) return fail(VTP_ERR_CUDA, cudaGetErrorString(e));
    // Global order of all rows by (scene, cell, attach id): fluid and boundary runs interleave.
    std::vector<uint32_t> scene_of(n, 0);
    for (auto &o : s->objs)
        for (uint32_t i = o.start; i < o.end; ++i) scene_of[i] = o.scene;
    std::vector<uint32_t> idx(n);
    std::iota(idx.begin(), idx.end(), 0u);
    std::sort(idx.begin(), idx.end(), [&](uint32_t a, uint32_t b) {
        const uint32_t sa = scene_of[ids[a]], sb = scene_of[ids[b]];
        if (sa != sb) return sa < sb;
        return keys[a] != keys[b] ? keys[a] < keys[b] : ids[a] < ids[b];
    });
    for (uint32_t k = 0; k < n; ++k) {
        sorted_ids[k] = ids[idx[k]];
        cell_ids[k] = keys[idx[k]];
    }
    return VTP_OK;
}

int vtp_solver_get_stage_times(vtp_solver *s, float *ms3) {
    if (!s || !ms3) return fail(VTP_ERR_ARG, "null argument");
    for (int k = 0; k < 3; ++k) ms3[k] = s->stage_ms[k];
    return VTP_OK;
}

int vtp_solver_profile_kernels(vtp_solver *s, uint32_t n, vtp_kernel_time *out, uint32_t cap, uint32_t *count) {
    if (!s || !out || !count) return fail(VTP_ERR_ARG, "null argument");
    int rc = VTP_OK;
    if (!s->initialized && (rc = s->initialize())) return rc;
    if (s->crashed) return fail(VTP_NOT_CONVERGED, "solver is crashed");
    auto P = std::make_unique<vtp::Profiler>();
    P->st = s->st;
    for (int k = 0; k < vtp::Profiler::kMax; ++k) {
        CU(cudaEventCreate(&P->beg[k]));
        CU(cudaEventCreate(&P->end[k]));
    }
    P->ready = true;
    const bool saved_loop = s->device_loop;
    s->device_loop = false;
    s->prof = P.get();
    if (s->type != VTP_SOLVER_PBF) {
        CU(cudaMemsetAsync(s->solve, 0, 2 * s->scenes.size() * sizeof(vtp::SolveState), s->st));
        CU(cudaMemsetAsync(s->loop, 0, 2 * sizeof(vtp::LoopState), s->st));
    }
    for (uint32_t k = 0; k < n && rc == VTP_OK; ++k) {
        rc = s->enqueue_tick(s->st, false);
        s->sim_time += s->dt;
        ++s->steps_done;
    }
    s->prof = nullptr;
    s->device_loop = saved_loop;
    cudaError_t e = cudaStreamSynchronize(s->st);
    std::vector<std::string> names;
    std::vector<float> tot;
    std::vector<uint32_t> cnt;
    for (int k = 0; k < P->n && e == cudaSuccess; ++k) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, P->beg[k], P->end[k]);
        size_t idx = std::find(names.begin(), names.end(), std::string(P->names[k])) - names.begin();
        if (idx == names.size()) names.push_back(P->names[k]), tot.push_back(0.f), cnt.push_back(0);
        tot[idx] += ms;
        cnt[idx] += 1;
    }
    for (int k = 0; k < vtp::Profiler::kMax; ++k) cudaEventDestroy(P->beg[k]), cudaEventDestroy(P->end[k]);
    if (e != cudaSuccess) return fail(VTP_ERR_CUDA, cudaGetErrorString(e));
    if (rc) return rc;
    uint32_t m = (uint32_t)std::min<size_t>(cap, names.size());
    for (uint32_t k = 0; k < m; ++k) {
        memset(out[k].name, 0, sizeof(out[k].name));
        strncpy(out[k].name, names[k].c_str(), sizeof(out[k].name) - 1);
        out[k].total_ms = tot[k];
        out[k].launches = cnt[k];
    }
    *count = m;
    s->stats.steps_done = s->steps_done;
    return s->check_status();
}

int vtp_solver_get_launch_count(vtp_solver *s, uint64_t *launches) {
    if (!s || !launches) return fail(VTP_ERR_ARG, "null argument");
    *launches = s->last_launches;
    return VTP_OK;
}

}  // extern "C"
