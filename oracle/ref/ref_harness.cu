// Harness that drives the reference's own solvers (compiled unmodified from
// their sources by oracle/ref/build_ref.py) through their public Solver API
// and reads their device state back.  Test infrastructure: it produces the
// golden vectors under tests/golden/ and is the reference arm of bench.py.
//
// Private members are reached by compiling the solver headers with
// `private`/`protected` mapped to `public` in this translation unit only.
#include <cstdint>
#include <cstring>
#include <fstream>
#include <iostream>
#include <map>
#include <memory>
#include <set>
#include <sstream>
#include <string>
#include <unordered_map>
#include <vector>

#include <cuda_runtime.h>
#include <vector_types.h>

#include "nlohmann/json.hpp"
#include "spdlog/spdlog.h"

#define private public
#define protected public
#include "Solvers/DFSPH/DFSPHSolver.hpp"
#include "Solvers/IMM-CT/IMMCTSolver.hpp"
#include "Solvers/IMM/IMMSolver.hpp"
#include "Solvers/PBF/PBFSolver.hpp"
#undef private
#undef protected
#include "Framework/Object.hpp"
#include "Framework/ObjectComponents.hpp"
#include "Model/ExportUtil.hpp"
#include "Model/ModelHandler.hpp"

using json = nlohmann::json;

// ---------------------------------------------------------------------------
// cal_mean (Simulator/Library/Source/DataAnalysis/CommonFunc.cpp:10-21),
// restated here so the harness can record each residual the solver loops
// compute: same work (copy of the whole array to the host, serial FP32 sum
// over [start, start + size)).
namespace {
std::vector<float> g_means;
}

namespace VT_Physics {
template <typename T>
T cal_mean(T *d_ptr, unsigned raw_size, unsigned target_size, unsigned target_start) {
    std::vector<T> data(raw_size);
    cudaMemcpy(data.data(), d_ptr, raw_size * sizeof(T), cudaMemcpyDeviceToHost);
    T mean = data[0] * 0;
    for (unsigned i = target_start; i < target_start + target_size; ++i) mean += data[i];
    return mean / target_size;
}

template <>
float cal_mean<float>(float *d_ptr, unsigned raw_size, unsigned target_size, unsigned target_start) {
    std::vector<float> data(raw_size);
    cudaMemcpy(data.data(), d_ptr, raw_size * sizeof(float), cudaMemcpyDeviceToHost);
    float mean = data[0] * 0;
    for (unsigned i = target_start; i < target_start + target_size; ++i) mean += data[i];
    float m = mean / target_size;
    g_means.push_back(m);
    return m;
}

template float3 cal_mean<float3>(float3 *, unsigned, unsigned, unsigned);
}  // namespace VT_Physics

using namespace VT_Physics;

namespace {

struct Entry {
    int type = 0;
    std::unique_ptr<Solver> solver;
    std::vector<std::unique_ptr<Object>> objs;
    long long next_id = 1;
};

std::map<int, Entry> g_solvers;
int g_next = 1;

Entry *get(int h) {
    auto it = g_solvers.find(h);
    return it == g_solvers.end() ? nullptr : &it->second;
}

template <class S>
int copy_field(S *s, const std::string &f, void *out, size_t bytes) {
    auto *d = s->m_host_data;
    auto &ns = s->m_neighborSearcher;
    const void *src = nullptr;
    size_t n = d->particle_num;
    size_t need = 0;
    if (f == "pos") src = d->pos, need = n * 12;
    else if (f == "vel") src = d->vel, need = n * 12;
    else if (f == "mass") src = d->mass, need = n * 4;
    else if (f == "volume") src = d->volume, need = n * 4;
    else if (f == "neighbors") src = ns.m_params_hostData.neighbors_cuData, need = n * ns.m_config_hostData.maxNeighborNum * 4;
    else if (f == "neighborNum") src = ns.m_params_hostData.neighborNum_cuData, need = n * 4;
    else if (f == "particleIndices") src = ns.m_params_hostData.particleIndices_cuData, need = n * 4;
    else if (f == "cellIndices") src = ns.m_params_hostData.cellIndices_cuData, need = n * 4;
    else {
        if constexpr (std::is_same<S, pbf::PBFSolver>::value) {
            if (f == "density_sph") src = d->density_sph, need = n * 4;
            else if (f == "lamb") src = d->lamb, need = n * 4;
        } else {
            if (f == "compression_ratio") src = d->compression_ratio, need = n * 4;
            else if (f == "df_alpha") src = d->df_alpha, need = n * 4;
            else if (f == "kappa_div") src = d->kappa_div, need = n * 4;
            else if (f == "kappa_incomp") src = d->kappa_incomp, need = n * 4;
            else if (f == "rest_density") src = d->rest_density, need = n * 4;
            else if (f == "delta_compression_ratio") src = d->delta_compression_ratio, need = n * 4;
            else if (f == "vel_adv") src = d->vel_adv, need = n * 12;
            if constexpr (std::is_same<S, immct::IMMCTSolver>::value || std::is_same<S, imm::IMMSolver>::value) {
                size_t P = d->phase_num;
                if (f == "vol_frac") src = d->vol_frac, need = n * P * 4;
                else if (f == "vel_phase") src = d->vel_phase, need = n * P * 12;
                else if (f == "vel_drift_phase") src = d->vel_drift_phase, need = n * P * 12;
            }
            if constexpr (std::is_same<S, immct::IMMCTSolver>::value) {
                if (f == "Q") src = d->Q, need = n * 36;
                else if (f == "vel_grad") src = d->vel_grad, need = n * 36;
                else if (f == "vise_stress") src = d->vise_stress, need = n * 36;
                else if (f == "Cd") src = d->Cd, need = n * 4;
            }
        }
    }
    if (!src) return -2;
    // pos / vel may be read for a leading range of particles (attach order), the rest whole
    const bool prefix_ok = (f == "pos" || f == "vel") && bytes <= need && bytes % 12 == 0;
    if (need != bytes && !prefix_ok) return -3;
    return cudaMemcpy(out, src, bytes, cudaMemcpyDeviceToHost) == cudaSuccess ? 0 : -4;
}

template <class S>
int set_field(S *s, const std::string &f, const void *in, size_t bytes) {
    auto *d = s->m_host_data;
    size_t n = d->particle_num;
    void *dst = nullptr;
    if (f == "pos") dst = d->pos;
    else if (f == "vel") dst = d->vel;
    if (!dst || bytes > n * 12 || bytes % 12) return -2;   // the leading particles (attach order)
    return cudaMemcpy(dst, in, bytes, cudaMemcpyHostToDevice) == cudaSuccess ? 0 : -4;
}

template <class S>
void override_velocity(S *s, size_t first, const float *vel, size_t n) {
    for (size_t i = 0; i < n; ++i) s->m_host_vel[first + i] = make_float3(vel[3 * i], vel[3 * i + 1], vel[3 * i + 2]);
}

template <class S>
size_t host_count(S *s) {
    return s->m_host_pos.size();
}

}  // namespace

extern "C" {

int ref_create(int type, const char *cfg_json) {
    Entry e;
    e.type = type;
    int dev = 0;
    cudaDeviceProp prop{};
    cudaGetDevice(&dev);
    cudaGetDeviceProperties(&prop, dev);
    const uint32_t threads = prop.maxThreadsPerBlock;  // SolverManager.cpp:11-17
    switch (type) {
        case 0: e.solver.reset(new pbf::PBFSolver(threads)); break;
        case 1: e.solver.reset(new dfsph::DFSPHSolver(threads)); break;
        case 2: e.solver.reset(new imm::IMMSolver(threads)); break;
        case 3: e.solver.reset(new immct::IMMCTSolver(threads)); break;
        default: return -1;
    }
    json cfg = json::parse(cfg_json);
    if (!e.solver->setConfig(cfg)) return -2;
    int h = g_next++;
    g_solvers[h] = std::move(e);
    return h;
}

int ref_attach(int h, const float *pos, uint32_t n, const float *vel, const char *obj_json) {
    Entry *e = get(h);
    if (!e) return -1;
    json o = json::parse(obj_json);
    auto obj = std::make_unique<Object>(e->next_id++);
    obj->transferTo(Particle_Common);
    obj->getObjectComponentConfig() = o["ObjectComponentConfig"];
    obj->attachSpecificSolverObjectComponentConfig(o["SolverObjectComponentConfig"]);
    if (o.contains("name")) obj->rename(o["name"].get<std::string>());
    auto *geo = static_cast<ParticleGeometryComponent *>(obj->getObjectComponent());
    geo->pos.assign(reinterpret_cast<const float3 *>(pos), reinterpret_cast<const float3 *>(pos) + n);
    size_t first = 0;
    switch (e->type) {
        case 0: first = host_count(static_cast<pbf::PBFSolver *>(e->solver.get())); break;
        case 1: first = host_count(static_cast<dfsph::DFSPHSolver *>(e->solver.get())); break;
        case 2: first = host_count(static_cast<imm::IMMSolver *>(e->solver.get())); break;
        case 3: first = host_count(static_cast<immct::IMMCTSolver *>(e->solver.get())); break;
    }
    if (!e->solver->attachObject(obj.get())) return -2;
    if (vel) {
        switch (e->type) {
            case 0: override_velocity(static_cast<pbf::PBFSolver *>(e->solver.get()), first, vel, n); break;
            case 1: override_velocity(static_cast<dfsph::DFSPHSolver *>(e->solver.get()), first, vel, n); break;
            case 2: override_velocity(static_cast<imm::IMMSolver *>(e->solver.get()), first, vel, n); break;
            case 3: override_velocity(static_cast<immct::IMMCTSolver *>(e->solver.get()), first, vel, n); break;
        }
    }
    e->objs.push_back(std::move(obj));
    return 0;
}

int ref_initialize(int h) {
    Entry *e = get(h);
    if (!e) return -1;
    if (!e->solver->initialize()) return -2;
    return cudaDeviceSynchronize() == cudaSuccess ? 0 : -4;
}

int ref_tick(int h, uint32_t n) {
    Entry *e = get(h);
    if (!e) return -1;
    bool ok = e->solver->tickNsteps(n);
    if (cudaDeviceSynchronize() != cudaSuccess) return -4;
    return ok ? 0 : -2;
}

// tickNsteps(n) bracketed by CUDA events on the legacy default stream (the
// stream every reference kernel uses); returns milliseconds, negative on error.
float ref_tick_timed(int h, uint32_t n) {
    Entry *e = get(h);
    if (!e) return -1.f;
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    cudaDeviceSynchronize();
    cudaEventRecord(a, 0);
    bool ok = e->solver->tickNsteps(n);
    cudaEventRecord(b, 0);
    cudaEventSynchronize(b);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    if (cudaGetLastError() != cudaSuccess) return -4.f;
    return ok ? ms : -2.f;
}

int ref_get(int h, const char *field, void *out, size_t bytes) {
    Entry *e = get(h);
    if (!e) return -1;
    std::string f(field);
    switch (e->type) {
        case 0: return copy_field(static_cast<pbf::PBFSolver *>(e->solver.get()), f, out, bytes);
        case 1: return copy_field(static_cast<dfsph::DFSPHSolver *>(e->solver.get()), f, out, bytes);
        case 2: return copy_field(static_cast<imm::IMMSolver *>(e->solver.get()), f, out, bytes);
        case 3: return copy_field(static_cast<immct::IMMCTSolver *>(e->solver.get()), f, out, bytes);
    }
    return -1;
}

int ref_set(int h, const char *field, const void *in, size_t bytes) {
    Entry *e = get(h);
    if (!e) return -1;
    std::string f(field);
    switch (e->type) {
        case 0: return set_field(static_cast<pbf::PBFSolver *>(e->solver.get()), f, in, bytes);
        case 1: return set_field(static_cast<dfsph::DFSPHSolver *>(e->solver.get()), f, in, bytes);
        case 2: return set_field(static_cast<imm::IMMSolver *>(e->solver.get()), f, in, bytes);
        case 3: return set_field(static_cast<immct::IMMCTSolver *>(e->solver.get()), f, in, bytes);
    }
    return -1;
}

// Residual means recorded by cal_mean since the last call (one per fluid
// object per solver iteration, in call order).
uint32_t ref_take_means(float *out, uint32_t cap) {
    uint32_t n = (uint32_t)g_means.size();
    if (out)
        for (uint32_t i = 0; i < n && i < cap; ++i) out[i] = g_means[i];
    g_means.clear();
    return n;
}

uint32_t ref_means_pending(void) { return (uint32_t)g_means.size(); }

// ModelHandler::generateObjectElements (ModelHandler.cpp:13-41) for a generator config
// (genType 1 sphere, 2 cube, 3 cylinder, 4 plane, 5 box): writes up to `cap` particles
// (x, y, z) into `out` and returns the count, or -1 on a bad config.  Host code only.
int64_t ref_generate(const char *cfg_json, float *out, int64_t cap) {
    json c;
    try {
        c = json::parse(cfg_json);
    } catch (...) {
        return -1;
    }
    const std::vector<float3> v = VT_Physics::ModelHandler::generateObjectElements(c);
    for (int64_t i = 0; out && i < (int64_t)v.size() && i < cap; ++i) {
        out[3 * i] = v[i].x;
        out[3 * i + 1] = v[i].y;
        out[3 * i + 2] = v[i].z;
    }
    return (int64_t)v.size();
}

// ExportUtil::exportData (ExportUtil.cpp:9-88) of n particles: positions, optional colors
// (n x 3) and phase fractions (n x nphase), to the path that function forms from `dir` and
// `name` (directory, a backslash, name, ".ply").  Host code only.
int ref_export_ply(const char *dir, const char *name, const float *pos, int64_t n, const float *color,
                   const float *phase, int nphase) {
    json c = {{"Common", {{"exportTargetDir", dir}, {"exportFilePrefix", name}, {"exportFileType", "PLY"}}}};
    if (phase) c["Common"]["exportPhaseNum"] = nphase;
    std::vector<float3> p((size_t)n), col;
    std::vector<float> ph;
    for (int64_t i = 0; i < n; ++i) p[i] = make_float3(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]);
    if (color) {
        col.resize((size_t)n);
        for (int64_t i = 0; i < n; ++i) col[i] = make_float3(color[3 * i], color[3 * i + 1], color[3 * i + 2]);
    }
    if (phase) ph.assign(phase, phase + n * nphase);
    VT_Physics::ExportUtil::exportData(c, p, col, ph);
    return 0;
}

int ref_destroy(int h) {
    Entry *e = get(h);
    if (!e) return -1;
    e->solver->destroy();
    g_solvers.erase(h);
    return 0;
}

}  // extern "C"
