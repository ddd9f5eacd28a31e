// PLY export of the solver state, as the reference's solvers write it
// (PBFSolver::exportData PBFSolver.cpp:248-324, DFSPHSolver.cpp:261-337,
// IMMCTSolver.cpp:320-406, IMMSolver.cpp, written by ExportUtil::exportAsPly
// ExportUtil.cpp:28-88): ASCII PLY, one vertex per particle in attach order,
// "x y z [r g b] [p1 .. pk] " per line with the default iostream float format.
//
// Trigger (PBFSolver.cpp:364-368 and the other ticks): after a substep,
// frame = frame + 1 whenever simTime >= frame / exportFps (FP32), and the
// file of that frame is written, when EXPORT.SolverRequired.enable is true.
//
// Policies:
//   MERGE: one file per exported material ("Fluid" / "Boundary") holding every
//          object of that material, at <dir>/<Material>/<frame>.ply; PBF and
//          DFSPH write positions only, IMM / IMM-CT add color and the phase
//          fractions.
//   SPLIT: one file per object whose exportFlag is set, at
//          <dir>/<object name>/<prefix><frame>.ply, positions and color.
// Two deliberate differences: the file path joins directory and name with '/'
// (the reference joins them with a backslash, ExportUtil.cpp:52, which on
// Linux names a file "dir\name.ply" beside an empty directory), and the
// merged phase fractions of the second and later objects are their own (the
// reference offsets vol_frac by the particle index instead of index x phases,
// IMMCTSolver.cpp:353-356).
#include "immct.h"
#include "solver.h"

#include <filesystem>
#include <fstream>
#include <set>
#include <string>
#include <vector>

using vtp::fail;

namespace {

int write_ply(const std::string &dir, const std::string &name, const std::vector<float> &pos,
              const std::vector<float> *color, const std::vector<float> *phase, int nphase) {
    std::error_code ec;
    std::filesystem::create_directories(dir, ec);
    if (ec) return fail(VTP_ERR_ARG, "cannot create export directory " + dir + ": " + ec.message());
    const std::string path = dir + "/" + name + ".ply";
    std::ofstream f(path);
    if (!f) return fail(VTP_ERR_ARG, "cannot open " + path);
    const size_t n = pos.size() / 3;
    f << "ply\n";
    f << "format ascii 1.0\n";
    f << "element vertex " << n << "\n";
    f << "property float x\n";
    f << "property float y\n";
    f << "property float z\n";
    if (color) {
        f << "property uchar red" << std::endl;
        f << "property uchar green" << std::endl;
        f << "property uchar blue" << std::endl;
    }
    if (phase)
        for (int k = 0; k < nphase; ++k) f << "property float p" << k + 1 << std::endl;
    f << "end_header\n";
    for (size_t i = 0; i < n; ++i) {
        f << pos[3 * i] << " " << pos[3 * i + 1] << " " << pos[3 * i + 2] << " ";
        if (color) f << (*color)[3 * i] << " " << (*color)[3 * i + 1] << " " << (*color)[3 * i + 2] << " ";
        if (phase)
            for (int k = 0; k < nphase; ++k) f << (*phase)[i * (size_t)nphase + k] << " ";
        f << "\n";
    }
    f.close();
    if (!f) return fail(VTP_ERR_ARG, "write failed: " + path);
    return VTP_OK;
}

}  // namespace

int vtp_solver::export_frame() {
    const vtp::NvtxRange nvtx_range("vtp export");
    const nlohmann::json &ex = cfg["EXPORT"];
    const std::string policy = ex["SolverRequired"]["exportGroupPolicy"].get<std::string>();
    const std::string dir = ex["Common"]["exportTargetDir"].get<std::string>();
    const std::string prefix = ex["Common"]["exportFilePrefix"].get<std::string>();
    const std::string ftype = ex["Common"].value("exportFileType", std::string("PLY"));
    if (ftype != "PLY") return fail(VTP_ERR_CONFIG, "Export type not supported.");
    const uint32_t n = L.n;
    std::vector<float> pos((size_t)n * 3), color((size_t)n * 3), phase;
    int rc;
    if ((rc = get_field(VTP_FIELD_POS, pos.data(), pos.size() * 4))) return rc;
    if ((rc = get_field(VTP_FIELD_COLOR, color.data(), color.size() * 4))) return rc;
    const bool mix = imm != nullptr;
    const int P = mix ? immct_phase_count(*this) : 0;
    if (mix) {
        phase.resize((size_t)n * P);
        if ((rc = get_field(VTP_FIELD_VOL_FRAC, phase.data(), phase.size() * 4))) return rc;
    }
    auto slice = [](const std::vector<float> &v, uint32_t a, uint32_t b, int w) {
        return std::vector<float>(v.begin() + (size_t)a * w, v.begin() + (size_t)b * w);
    };
    const std::string frame = std::to_string(out_frames);
    if (policy == "MERGE") {
        std::set<int> done;
        for (const ObjRec &o : objs) {
            if (!o.export_flag || done.count(o.mat)) continue;
            done.insert(o.mat);
            std::vector<float> p, c, ph;
            // every object of that material is merged (PBFSolver.cpp:260-275)
            for (const ObjRec &q : objs) {
                if (q.mat != o.mat) continue;
                auto a = slice(pos, q.start, q.end, 3), b = slice(color, q.start, q.end, 3);
                p.insert(p.end(), a.begin(), a.end());
                c.insert(c.end(), b.begin(), b.end());
                if (mix) {
                    auto f = slice(phase, q.start, q.end, P);
                    ph.insert(ph.end(), f.begin(), f.end());
                }
            }
            const std::string sub = dir + "/" + (o.mat == 0 ? "Fluid" : "Boundary");
            if ((rc = write_ply(sub, frame, p, mix ? &c : nullptr, mix ? &ph : nullptr, P))) return rc;
        }
    } else if (policy == "SPLIT") {
        for (const ObjRec &o : objs) {
            if (!o.export_flag) continue;
            auto p = slice(pos, o.start, o.end, 3), c = slice(color, o.start, o.end, 3);
            if ((rc = write_ply(dir + "/" + o.name, prefix + frame, p, &c, nullptr, 0))) return rc;
        }
    } else {
        return fail(VTP_ERR_CONFIG, std::string("exportGroupPolicy ") + policy + " not supported.");
    }
    ++frames_written;
    return VTP_OK;
}

int vtp_solver::maybe_export() {
    // PBFSolver::tick (PBFSolver.cpp:364-368): the frame counter advances when the FP32
    // simulated time passes frame / exportFps; tickNsteps / run then export that frame.
    if (!export_enabled) return VTP_OK;
    if (sim_time >= export_gap * (float)out_frames) {
        ++out_frames;
        cudaError_t e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return fail(VTP_ERR_CUDA, cudaGetErrorString(e));
        return export_frame();
    }
    return VTP_OK;
}
