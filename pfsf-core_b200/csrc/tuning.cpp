// Launch-shape and smoother parameters of the batched tolerance solve: the
// tuning file written by the autotuner (pfsf_b200/autotune.py), environment
// overrides, and the pfsf_get_tuning / pfsf_set_tuning exports.
//
// File format (text): '#' comments, one section per GPU model,
//     [<device name> <SM count>]
//     cluster = 4
//     cluster_min_voxels = 262144
//     ...
// The engine takes the section whose name and SM count match its device.
#include <dlfcn.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <string>

#include "engine.h"

namespace pfsf_b200 {

namespace {

std::string trim(const std::string& s) {
    const size_t a = s.find_first_not_of(" \t\r\n");
    if (a == std::string::npos) return "";
    const size_t b = s.find_last_not_of(" \t\r\n");
    return s.substr(a, b - a + 1);
}

// the solver parameters are part of a caller's struct only when its size covers them
bool has_solver(const pfsf_tuning& t) { return t.struct_bytes >= (int32_t)sizeof(pfsf_tuning); }

bool valid(const pfsf_tuning& t) {
    const bool launch = (t.cluster == 1 || t.cluster == 4 || t.cluster == 8) && t.cluster_min_voxels >= 0 &&
                        t.grid_min_voxels >= 0 && t.warp_max_voxels >= 0 && t.cheb_k >= 1 && t.cheb_k <= 4;
    const bool solver = !has_solver(t) || (t.cheb_lower > 0.0f && t.cheb_lower < 1.0f && t.coarse_weight > 0.0f &&
                                           t.coarse_weight < 2.0f && t.tail_cells >= 0 && t.tail_cells <= (1 << 20) &&
                                           t.coarse_sweeps >= 1 && t.coarse_sweeps <= 16 && t.inner_eta > 1e-6f &&
                                           t.inner_eta < 1.0f);
    return launch && solver;
}

// tune/pfsf_tune.txt beside the directory that holds this library
std::string default_tuning_path() {
    Dl_info info{};
    if (!dladdr(reinterpret_cast<void*>(&default_tuning_path), &info) || !info.dli_fname) return "";
    std::string lib = info.dli_fname;
    const size_t a = lib.rfind('/');
    if (a == std::string::npos) return "";
    const std::string libdir = lib.substr(0, a);
    const size_t b = libdir.rfind('/');
    const std::string root = b == std::string::npos ? "." : libdir.substr(0, b);
    return root + "/tune/pfsf_tune.txt";
}

}  // namespace

void Engine::load_tuning() {
    pfsf_tuning t{};
    get_tuning(&t);
    const char* env = std::getenv("PFSF_TUNE_FILE");
    const std::string path = env ? std::string(env) : default_tuning_path();
    cudaDeviceProp prop{};
    std::string want;
    if (cudaGetDeviceProperties(&prop, device_) == cudaSuccess)
        want = std::string(prop.name) + " " + std::to_string(prop.multiProcessorCount);
    else
        cudaGetLastError();
    std::ifstream in(path);
    bool in_section = false, found = false;
    std::string line;
    while (!want.empty() && in && std::getline(in, line)) {
        line = trim(line);
        if (line.empty() || line[0] == '#') continue;
        if (line.front() == '[' && line.back() == ']') {
            in_section = trim(line.substr(1, line.size() - 2)) == want;
            found |= in_section;
            continue;
        }
        if (!in_section) continue;
        const size_t eq = line.find('=');
        if (eq == std::string::npos) continue;
        const std::string k = trim(line.substr(0, eq));
        const long long v = std::atoll(trim(line.substr(eq + 1)).c_str());
        if (k == "cluster") t.cluster = (int32_t)v;
        else if (k == "cluster_min_voxels") t.cluster_min_voxels = v;
        else if (k == "grid_min_voxels") t.grid_min_voxels = v;
        else if (k == "warp_max_voxels") t.warp_max_voxels = v;
        else if (k == "cheb_k") t.cheb_k = (int32_t)v;
        else if (k == "cheb_lower") t.cheb_lower = std::strtof(trim(line.substr(eq + 1)).c_str(), nullptr);
        else if (k == "coarse_weight") t.coarse_weight = std::strtof(trim(line.substr(eq + 1)).c_str(), nullptr);
        else if (k == "tail_cells") t.tail_cells = (int32_t)v;
        else if (k == "coarse_sweeps") t.coarse_sweeps = (int32_t)v;
        else if (k == "inner_eta") t.inner_eta = std::strtof(trim(line.substr(eq + 1)).c_str(), nullptr);
    }
    if (found && valid(t)) {
        set_tuning(&t);
        tuning_source_ = PFSF_TUNING_FILE;
    } else if (found) {
        std::fprintf(stderr, "[libpfsf] tuning file %s: section [%s] out of range; defaults kept\n", path.c_str(),
                     want.c_str());
    }
    bool over = false;
    if (const char* f = std::getenv("PFSF_CLUSTER_MIN_VOXELS")) { cluster_min_voxels_ = std::atoll(f); over = true; }
    if (const char* f = std::getenv("PFSF_GRID_MIN_VOXELS")) { grid_min_voxels_ = std::atoll(f); over = true; }
    if (const char* f = std::getenv("PFSF_CLUSTER")) { cluster_size_ = std::atoi(f); over = true; }
    if (const char* f = std::getenv("PFSF_WARP_MAX_VOXELS")) { warp_max_voxels_ = std::atoll(f); over = true; }
    if (const char* f = std::getenv("PFSF_CHEB_K")) { cheb_k_ = std::atoi(f); over = true; }
    if (const char* f = std::getenv("PFSF_CHEB_LOWER")) { cheb_lower_ = std::strtof(f, nullptr); over = true; }
    if (const char* f = std::getenv("PFSF_COARSE_WEIGHT")) { coarse_weight_ = std::strtof(f, nullptr); over = true; }
    if (const char* f = std::getenv("PFSF_TAIL_CELLS")) { tail_cells_ = std::atoi(f); over = true; }
    if (const char* f = std::getenv("PFSF_COARSE_SWEEPS")) { coarse_sweeps_ = std::atoi(f); over = true; }
    if (const char* f = std::getenv("PFSF_INNER_ETA")) { inner_eta_ = std::strtof(f, nullptr); over = true; }
    if (over) tuning_source_ = PFSF_TUNING_ENV;
}

pfsf_result Engine::get_tuning(pfsf_tuning* out) const {
    if (!out) return PFSF_ERROR_INVALID_ARG;
    pfsf_tuning t{};
    t.struct_bytes = (int32_t)sizeof(t);
    t.cluster = cluster_size_;
    t.cluster_min_voxels = cluster_min_voxels_;
    t.grid_min_voxels = grid_min_voxels_;
    t.warp_max_voxels = warp_max_voxels_;
    t.cheb_k = cheb_k_;
    t.source = tuning_source_;
    t.cheb_lower = cheb_lower_;
    t.coarse_weight = coarse_weight_;
    t.tail_cells = tail_cells_;
    t.coarse_sweeps = coarse_sweeps_;
    t.inner_eta = inner_eta_;
    // a caller's older, shorter struct gets the fields it has
    const size_t n = out->struct_bytes > 0 ? std::min(sizeof(t), (size_t)out->struct_bytes) : sizeof(t);
    std::memcpy(out, &t, n);
    return PFSF_OK;
}

pfsf_result Engine::set_tuning(const pfsf_tuning* in) {
    if (!in || !valid(*in)) return PFSF_ERROR_INVALID_ARG;
    cluster_size_ = in->cluster;
    cluster_min_voxels_ = in->cluster_min_voxels;
    grid_min_voxels_ = in->grid_min_voxels;
    warp_max_voxels_ = in->warp_max_voxels;
    cheb_k_ = in->cheb_k;
    if (has_solver(*in)) {
        cheb_lower_ = in->cheb_lower;
        coarse_weight_ = in->coarse_weight;
        tail_cells_ = in->tail_cells;
        coarse_sweeps_ = in->coarse_sweeps;
        inner_eta_ = in->inner_eta;
    }
    tuning_source_ = PFSF_TUNING_CALLER;
    return PFSF_OK;
}

}  // namespace pfsf_b200
