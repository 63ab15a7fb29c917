// Checkpoint writer and reader in the reference's file layout
// (ComputeUnitBase::checkpoint_write / checkpoint_read, ComputeUnit.hpp:318-439;
// file names DiskOutputTree.h:572-589):
//
//   <dir>/checkpoint_grid.<idi>.<idj>.<idk>.<unit>.Q    xg*yg*zg x 18 float (QVec, AoS)
//   <dir>/checkpoint_grid.<idi>.<idj>.<idk>.<unit>.F    xg*yg*zg x 3 float  (Force)
//   <dir>/checkpoint_grid.<idi>.<idj>.<idk>.<unit>.Nu   xg*yg*zg float
//   <dir>/AllParams.<idi>.<idj>.<idk>.<unit>.json       all params (DiskOutputTree.h:415-481)
//
// over the ghosted grid (xg = x + 2, index (i*yg + j)*zg + k). Q holds what
// the reference's Q holds between steps: the moments M01..M18 (after
// moments()), at the cell itself for Simple and, for Esotwist, where the
// writeMoments map puts them (StreamingEsoteric.hpp:131-179): moment d of
// cell x in slot d (even step) or d^1 (odd step) of cell x + max(-c_d, 0),
// wrapping over the interior. Ghost cells are written as zero (the
// reference's step never reads them); F is zero where the last forcing pass
// did not touch a cell, as the reference's is (Forcing.hpp:162-174).
//
// Extension: the reference does not store evenStep, so an Esotwist
// checkpoint written after an odd number of steps reads back with the wrong
// parity there. The params file here carries "StreamingState": {"evenStep"}
// and the reader uses it (absent: true, the reference's initial value).
//
// Reading needs FP32 storage (16-bit storage holds populations only);
// writing works for every storage. Both use a device scratch of the ghosted
// AoS Q (72 bytes per cell) for the transpose.
#include "tdlb_handle.hpp"
#include "step_kernels.cuh"

#include <nlohmann/json.hpp>

#include <sys/stat.h>
#include <sys/types.h>

#include <algorithm>
#include <cerrno>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

namespace tdlb {

__device__ __forceinline__ long long ghost_index(const Dims& g, int i, int j, int k) {
    return ((long long)(i + 1) * (g.ny + 2) + (j + 1)) * (long long)(g.nz + 2) + (k + 1);
}

// Q out: the moments of every interior cell, placed as the reference's Q
// holds them (see the file header).
template <typename S>
__global__ void __launch_bounds__(256) k_ckpt_q_out(Planes A, Dims g, int mode, int even, CollideParams p, int esotwist,
                                                    float* __restrict__ out) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= g.rows() * g.nz) return;
    const int k = (int)(t % g.nz);
    const long long row = t / g.nz;
    const int j = (int)(row % g.ny);
    const int i = (int)(row / g.ny);
    float m[NQ];
    state_moments18<S>(A, g, mode, even, p, i, j, k, m);
    if (!esotwist) {
        float* o = out + ghost_index(g, i, j, k) * NQ;
#pragma unroll
        for (int d = 0; d < NQ; d++) o[d] = m[d];
        return;
    }
    const int i1 = i + 1 == g.nx ? 0 : i + 1, j1 = j + 1 == g.ny ? 0 : j + 1, k1 = k + 1 == g.nz ? 0 : k + 1;
#pragma unroll
    for (int d = 0; d < NQ; d++) {
        const int li = cx_of(d) < 0 ? i1 : i, lj = cy_of(d) < 0 ? j1 : j, lk = cz_of(d) < 0 ? k1 : k;
        out[ghost_index(g, li, lj, lk) * NQ + (even ? d : (d ^ 1))] = m[d];
    }
}

__global__ void __launch_bounds__(256) k_ckpt_f_out(const float4* __restrict__ F, const uint32_t* __restrict__ mask,
                                                    const float* __restrict__ Nu, Dims g, float* __restrict__ f3,
                                                    float* __restrict__ nu) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= g.rows() * g.nz) return;
    const int k = (int)(t % g.nz);
    const long long row = t / g.nz;
    const int j = (int)(row % g.ny);
    const int i = (int)(row / g.ny);
    const long long e = row * g.kp + k;
    const long long o = ghost_index(g, i, j, k);
    const bool on = (mask[row * g.kw + (k >> 5)] >> (k & 31)) & 1u;
    const float4 v = F[e];
    f3[3 * o] = on ? v.x : 0.f;
    f3[3 * o + 1] = on ? v.y : 0.f;
    f3[3 * o + 2] = on ? v.z : 0.f;
    nu[o] = Nu[e];
}

// Q in: slot s of interior cell x goes to plane s at x, for both schemes (the
// state then holds moments: at the cell for Simple, in the read-map places
// of the stored parity for Esotwist).
__global__ void __launch_bounds__(256) k_ckpt_q_in(const float* __restrict__ in, Planes A, Dims g) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= g.rows() * g.nz) return;
    const int k = (int)(t % g.nz);
    const long long row = t / g.nz;
    const int j = (int)(row % g.ny);
    const int i = (int)(row / g.ny);
    const float* q = in + ghost_index(g, i, j, k) * NQ;
    const long long e = row * g.kp + k;
#pragma unroll
    for (int s = 0; s < NQ; s++) A.p[s][e] = q[s];
}

// F and Nu in; one thread per touched-flag word: a cell counts as touched
// where its F is non-zero (an untouched cell's F is zero, and a touched one
// whose F is exactly zero acts the same either way).
__global__ void __launch_bounds__(256) k_ckpt_f_in(const float* __restrict__ f3, const float* __restrict__ nu, Dims g,
                                                   float4* __restrict__ F, float* __restrict__ Nu,
                                                   uint32_t* __restrict__ mask) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= g.rows() * g.kw) return;
    const long long row = t / g.kw;
    const int w = (int)(t - row * g.kw);
    const int j = (int)(row % g.ny);
    const int i = (int)(row / g.ny);
    uint32_t bits = 0;
    for (int b = 0; b < 32; b++) {
        const int k = w * 32 + b;
        if (k >= g.kp) break;
        const long long e = row * g.kp + k;
        if (k >= g.nz) {
            F[e] = make_float4(0.f, 0.f, 0.f, 0.f);
            Nu[e] = 0.f;
            continue;
        }
        const long long o = ghost_index(g, i, j, k);
        const float x = f3[3 * o], y = f3[3 * o + 1], z = f3[3 * o + 2];
        F[e] = make_float4(x, y, z, 0.f);
        Nu[e] = nu[o];
        if (x != 0.f || y != 0.f || z != 0.f) bits |= 1u << b;
    }
    mask[t] = bits;
}

}  // namespace tdlb

namespace {

struct CFail {
    int code;
    std::string msg;
};

#define TDLB_CCK(call)                                                                                      \
    do {                                                                                                    \
        cudaError_t e_ = (call);                                                                            \
        if (e_ != cudaSuccess) throw CFail{TDLB_ECUDA, std::string(#call) + ": " + cudaGetErrorString(e_)}; \
    } while (0)

template <typename F>
int cguard(tdlb_lattice* h, F&& fn) {
    if (!h) return TDLB_EINVAL;
    try {
        cudaSetDevice(h->device);
        const cudaError_t je = tdlb_rt::join_side(h);   // after every queued step and forcing pass
        if (je != cudaSuccess) throw CFail{TDLB_ECUDA, std::string("join: ") + cudaGetErrorString(je)};
        fn();
        return TDLB_OK;
    } catch (const CFail& f) {
        h->err = f.msg;
        return f.code;
    } catch (const std::bad_alloc&) {
        h->err = "host allocation failed";
        return TDLB_ENOMEM;
    } catch (const std::exception& e) {
        h->err = e.what();
        return TDLB_EJSON;
    }
}

// Device scratch and pinned staging, freed on every exit path.
struct Scratch {
    float* dev = nullptr;
    char* pin = nullptr;
    ~Scratch() {
        cudaFree(dev);
        cudaFreeHost(pin);
    }
};

constexpr size_t kStage = (size_t)64 << 20;

std::string id_of(const nlohmann::json& all) {
    int idi = 0, idj = 0, idk = 0;
    if (all.contains("ComputeUnitParams") && all["ComputeUnitParams"].is_object()) {
        const auto& c = all["ComputeUnitParams"];
        idi = c.value("idi", 0);
        idj = c.value("idj", 0);
        idk = c.value("idk", 0);
    }
    return std::to_string(idi) + "." + std::to_string(idj) + "." + std::to_string(idk);
}

std::string grid_file(const std::string& dir, const std::string& id, const std::string& unit, const char* matrix) {
    return dir + "/checkpoint_grid." + id + "." + unit + "." + matrix;
}

std::string params_file(const std::string& dir, const std::string& id, const std::string& unit) {
    return dir + "/AllParams." + id + "." + unit;
}

void write_device(const std::string& path, const float* dev, size_t bytes, cudaStream_t st, char* pin) {
    FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) throw CFail{TDLB_EIO, "cannot write " + path + ": " + std::strerror(errno)};
    for (size_t off = 0; off < bytes; off += kStage) {
        const size_t n = std::min(kStage, bytes - off);
        const cudaError_t e = cudaMemcpyAsync(pin, reinterpret_cast<const char*>(dev) + off, n, cudaMemcpyDeviceToHost, st);
        const cudaError_t s = e == cudaSuccess ? cudaStreamSynchronize(st) : e;
        if (s != cudaSuccess) {
            std::fclose(f);
            throw CFail{TDLB_ECUDA, std::string("checkpoint copy: ") + cudaGetErrorString(s)};
        }
        if (std::fwrite(pin, 1, n, f) != n) {
            std::fclose(f);
            throw CFail{TDLB_EIO, "short write to " + path};
        }
    }
    if (std::fclose(f) != 0) throw CFail{TDLB_EIO, "cannot close " + path};
}

void read_device(const std::string& path, float* dev, size_t bytes, cudaStream_t st, char* pin) {
    FILE* f = std::fopen(path.c_str(), "rb");
    if (!f) throw CFail{TDLB_EIO, "checkpoint_read: file could not be read: " + path};
    std::fseek(f, 0, SEEK_END);
    const long size = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    if (size < 0 || (size_t)size != bytes) {
        std::fclose(f);
        throw CFail{TDLB_EIO, path + ": " + std::to_string(size) + " bytes, expected " + std::to_string(bytes)};
    }
    for (size_t off = 0; off < bytes; off += kStage) {
        const size_t n = std::min(kStage, bytes - off);
        if (std::fread(pin, 1, n, f) != n) {
            std::fclose(f);
            throw CFail{TDLB_EIO, "short read from " + path};
        }
        const cudaError_t e = cudaMemcpyAsync(reinterpret_cast<char*>(dev) + off, pin, n, cudaMemcpyHostToDevice, st);
        const cudaError_t s = e == cudaSuccess ? cudaStreamSynchronize(st) : e;
        if (s != cudaSuccess) {
            std::fclose(f);
            throw CFail{TDLB_ECUDA, std::string("checkpoint copy: ") + cudaGetErrorString(s)};
        }
    }
    std::fclose(f);
}

void ensure_dir(const std::string& dir) {
    struct stat sb;
    if (stat(dir.c_str(), &sb) == 0) {
        if (!S_ISDIR(sb.st_mode)) throw CFail{TDLB_EIO, dir + " is not a directory"};
        return;
    }
    if (mkdir(dir.c_str(), 0755) != 0 && errno != EEXIST)
        throw CFail{TDLB_EIO, "cannot create " + dir + ": " + std::strerror(errno)};
}

// The params file: the caller's sections (if any) completed with the
// reference's keys for everything the handle knows.
nlohmann::json all_params(const tdlb_lattice* h, const char* params_json, const std::string& bin_path, long long ng) {
    nlohmann::json all = nlohmann::json::object();
    if (params_json && *params_json) {
        all = nlohmann::json::parse(params_json);
        if (!all.is_object()) throw CFail{TDLB_EJSON, "params JSON must be an object"};
    }
    const tdlb_config& c = h->cfg;
    const bool eso = c.streaming == TDLB_STREAMING_ESOTWIST;
    auto section = [&](const char* name) -> nlohmann::json& {
        if (!all.contains(name) || !all[name].is_object()) all[name] = nlohmann::json::object();
        return all[name];
    };
    {   // Params/ComputeUnitParams.hpp:97-116
        auto& cu = section("ComputeUnitParams");
        const nlohmann::json defaults = {
            {"nodeID", 0}, {"deviceID", h->device}, {"idi", 0}, {"idj", 0}, {"idk", 0}, {"i0", 0}, {"j0", 0},
            {"k0", 0}, {"ghost", 1}, {"resolution", 1}, {"strQVecPrecision", "float"}, {"strQLength", "QLen::D3Q19"},
            {"strMemoryLayout", "MemoryLayoutIJKL"}, {"strCollisonAlgo", "EgglesSomers"},
            {"strStreamingAlgo", eso ? "Esotwist" : "Simple"}, {"strCompileFlag", "B200"}};
        for (auto it = defaults.begin(); it != defaults.end(); ++it)
            if (!cu.contains(it.key())) cu[it.key()] = it.value();
        cu["x"] = c.x; cu["y"] = c.y; cu["z"] = c.z;
    }
    {   // Params/GridParams.hpp:72-79
        auto& gr = section("GridParams");
        const nlohmann::json defaults = {{"ngx", 1}, {"ngy", 1}, {"ngz", 1}, {"strMinQVecPrecision", "float"}};
        for (auto it = defaults.begin(); it != defaults.end(); ++it)
            if (!gr.contains(it.key())) gr[it.key()] = it.value();
        gr["x"] = c.x; gr["y"] = c.y; gr["z"] = c.z; gr["multiStep"] = 1;
    }
    {   // Params/FlowParams.hpp:112-128; the handle's values win
        auto& fl = section("FlowParams");
        const nlohmann::json defaults = {{"reMNonDimensional", 0.0}, {"uav", 0.0}, {"fx0", 0.0}, {"fy0", 0.0},
                                         {"fz0", 0.0}, {"Re_m", 0.0}, {"Re_f", 0.0}, {"uf", 0.0},
                                         {"collision", "EgglesSomers"}};
        for (auto it = defaults.begin(); it != defaults.end(); ++it)
            if (!fl.contains(it.key())) fl[it.key()] = it.value();
        fl["initialRho"] = c.initialRho; fl["nu"] = c.nu; fl["cs0"] = c.cs0; fl["g3"] = c.g3;
        fl["alpha"] = c.alpha; fl["beta"] = c.beta; fl["useLES"] = c.useLES != 0;
        fl["streaming"] = eso ? "Esotwist" : "Simple";
    }
    {   // Params/RunningParams.hpp (the caller's, else the attached impeller's step)
        auto& rn = section("RunningParams");
        const nlohmann::json defaults = {
            {"step", (long long)h->rstep}, {"angle", h->angle}, {"num_steps", 0},
            {"impellerStartupStepsUntilNormalSpeed", (long long)h->rspec.startup_steps}, {"numStepsForAverageCalc", 10},
            {"repeatPrintTimerToFile", 20}, {"repeatPrintTimerToStdOut", 10}, {"runningDataFileDir", "."},
            {"runningDataFilePrefix", "debug"}, {"runningDataFileAppendTime", false}, {"doubleResolutionAtStep", 0}};
        for (auto it = defaults.begin(); it != defaults.end(); ++it)
            if (!rn.contains(it.key())) rn[it.key()] = it.value();
    }
    section("OutputParams");
    {   // Params/CheckpointParams.hpp:66-71
        auto& ck = section("CheckpointParams");
        const nlohmann::json defaults = {{"startWithCheckpoint", false}, {"checkpointLoadFromDir", ""},
                                         {"checkpointRepeat", 0}, {"checkpointWriteRootDir", "."},
                                         {"checkpointWriteDirPrefix", ""}, {"checkpointWriteDirAppendTime", false}};
        for (auto it = defaults.begin(); it != defaults.end(); ++it)
            if (!ck.contains(it.key())) ck[it.key()] = it.value();
    }
    // ComputeUnit.hpp:395-403
    all["BinFileParams"] = {{"filePath", bin_path}, {"name", ""}, {"note", ""}, {"structName", "checkpoint"},
                            {"binFileSizeInStructs", ng}, {"coordsType", "none"}, {"hasGridtCoords", false},
                            {"hasColRowtCoords", false}, {"reference", ""}, {"i0", 0}, {"j0", 0}, {"k0", 0},
                            {"QDataType", "none"}, {"QOutputLength", 18}};
    all["StreamingState"] = {{"evenStep", eso ? h->even : true}};
    return all;
}

long long ghost_cells(const Dims& g) { return (long long)(g.nx + 2) * (g.ny + 2) * (g.nz + 2); }

unsigned blocks(long long n) { return (unsigned)((n + 255) / 256); }

}  // namespace

extern "C" {

int tdlb_checkpoint_write(tdlb_handle h, const char* dir, const char* unit_name, const char* params_json) {
    return cguard(h, [&] {
        if (!h->initialised) throw CFail{TDLB_ESTATE, "not initialised (tdlb_initialise)"};
        if (!dir || !unit_name || !*unit_name) throw CFail{TDLB_EINVAL, "dir and unit_name are required"};
        nlohmann::json probe = nlohmann::json::object();
        if (params_json && *params_json) {
            try {
                probe = nlohmann::json::parse(params_json);
            } catch (const std::exception& e) {
                throw CFail{TDLB_EJSON, std::string("params JSON: ") + e.what()};
            }
        }
        const std::string sdir(dir), unit(unit_name), id = id_of(probe);
        const Dims& g = h->g;
        const long long ng = ghost_cells(g);
        const nlohmann::json all = all_params(h, params_json, params_file(sdir, id, unit), ng);
        ensure_dir(sdir);
        {
            FILE* f = std::fopen((params_file(sdir, id, unit) + ".json").c_str(), "wb");
            if (!f) throw CFail{TDLB_EIO, "cannot write " + params_file(sdir, id, unit) + ".json"};
            const std::string text = all.dump();
            const size_t n = std::fwrite(text.data(), 1, text.size(), f);
            std::fclose(f);
            if (n != text.size()) throw CFail{TDLB_EIO, "short write of the params file"};
        }
        Scratch sc;
        TDLB_CCK(cudaMalloc(&sc.dev, (size_t)ng * tdlb::NQ * sizeof(float)));
        TDLB_CCK(cudaHostAlloc((void**)&sc.pin, kStage, cudaHostAllocDefault));
        const long long cells = g.rows() * g.nz;
        const int eso = h->cfg.streaming == TDLB_STREAMING_ESOTWIST;
        // Q
        TDLB_CCK(cudaMemsetAsync(sc.dev, 0, (size_t)ng * tdlb::NQ * sizeof(float), h->stream));
        const Planes A = h->planes(h->state_buf());
        const int mode = h->state_mode(), even = h->even ? 1 : 0;
        tdlb::with_storage(h->cfg.storage, [&](auto s) {
            tdlb::k_ckpt_q_out<decltype(s)><<<blocks(cells), 256, 0, h->stream>>>(A, g, mode, even, h->cp, eso, sc.dev);
        });
        TDLB_CCK(cudaGetLastError());
        write_device(grid_file(sdir, id, unit, "Q"), sc.dev, (size_t)ng * tdlb::NQ * sizeof(float), h->stream, sc.pin);
        // F and Nu share the scratch: F at [0, 3 ng), Nu at [3 ng, 4 ng)
        TDLB_CCK(cudaMemsetAsync(sc.dev, 0, (size_t)ng * 4 * sizeof(float), h->stream));
        tdlb::k_ckpt_f_out<<<blocks(cells), 256, 0, h->stream>>>(reinterpret_cast<const float4*>(h->F), h->mask_cur(),
                                                                 h->Nu, g, sc.dev, sc.dev + 3 * ng);
        TDLB_CCK(cudaGetLastError());
        write_device(grid_file(sdir, id, unit, "F"), sc.dev, (size_t)ng * 3 * sizeof(float), h->stream, sc.pin);
        write_device(grid_file(sdir, id, unit, "Nu"), sc.dev + 3 * ng, (size_t)ng * sizeof(float), h->stream, sc.pin);
    });
}

int tdlb_checkpoint_read(tdlb_handle h, const char* dir, const char* unit_name) {
    return cguard(h, [&] {
        if (!dir || !unit_name || !*unit_name) throw CFail{TDLB_EINVAL, "dir and unit_name are required"};
        if (h->cfg.storage != TDLB_STORAGE_FP32)
            throw CFail{TDLB_EINVAL, "checkpoint_read needs FP32 storage (16-bit storage holds populations only)"};
        const std::string sdir(dir), unit(unit_name), id = "0.0.0";
        nlohmann::json all;
        {
            const std::string path = params_file(sdir, id, unit) + ".json";
            FILE* f = std::fopen(path.c_str(), "rb");
            if (!f) throw CFail{TDLB_EIO, "checkpoint_read: params file could not be read: " + path};
            std::string text;
            char buf[65536];
            size_t n;
            while ((n = std::fread(buf, 1, sizeof buf, f)) > 0) text.append(buf, n);
            std::fclose(f);
            try {
                all = nlohmann::json::parse(text);
            } catch (const std::exception& e) {
                throw CFail{TDLB_EJSON, path + ": " + e.what()};
            }
        }
        const Dims& g = h->g;
        tdlb_config c = h->cfg;
        try {   // the lattice shape must match; flow params are taken from the file (ComputeUnit.hpp:341)
            if (all.contains("ComputeUnitParams") && all["ComputeUnitParams"].is_object()) {
                const auto& cu = all["ComputeUnitParams"];
                if (cu.at("x").get<long long>() != c.x || cu.at("y").get<long long>() != c.y ||
                    cu.at("z").get<long long>() != c.z)
                    throw CFail{TDLB_EINVAL, "checkpoint lattice size differs from this handle's"};
            }
            if (all.contains("FlowParams") && all["FlowParams"].is_object()) {
                const auto& fl = all["FlowParams"];
                c.initialRho = fl.value("initialRho", c.initialRho);
                c.nu = fl.value("nu", c.nu);
                c.cs0 = fl.value("cs0", c.cs0);
                c.g3 = fl.value("g3", c.g3);
                c.alpha = fl.value("alpha", c.alpha);
                c.beta = fl.value("beta", c.beta);
                if (fl.contains("useLES")) c.useLES = fl["useLES"].get<bool>() ? 1 : 0;
            }
        } catch (const CFail&) {
            throw;
        } catch (const std::exception& e) {
            throw CFail{TDLB_EJSON, std::string("params file: ") + e.what()};
        }
        bool even = true;
        if (all.contains("StreamingState") && all["StreamingState"].is_object())
            even = all["StreamingState"].value("evenStep", true);
        const long long ng = ghost_cells(g);
        Scratch sc;
        TDLB_CCK(cudaMalloc(&sc.dev, (size_t)ng * tdlb::NQ * sizeof(float)));
        TDLB_CCK(cudaHostAlloc((void**)&sc.pin, kStage, cudaHostAllocDefault));
        const long long cells = g.rows() * g.nz;
        read_device(grid_file(sdir, id, unit, "Q"), sc.dev, (size_t)ng * tdlb::NQ * sizeof(float), h->stream, sc.pin);
        tdlb::k_ckpt_q_in<<<blocks(cells), 256, 0, h->stream>>>(sc.dev, h->planes(h->bufA), g);
        TDLB_CCK(cudaGetLastError());
        read_device(grid_file(sdir, id, unit, "F"), sc.dev, (size_t)ng * 3 * sizeof(float), h->stream, sc.pin);
        read_device(grid_file(sdir, id, unit, "Nu"), sc.dev + 3 * ng, (size_t)ng * sizeof(float), h->stream, sc.pin);
        TDLB_CCK(cudaMemsetAsync(h->mask, 0, (size_t)2 * h->mask_words * sizeof(uint32_t), h->stream));
        tdlb::k_ckpt_f_in<<<blocks(g.rows() * g.kw), 256, 0, h->stream>>>(sc.dev, sc.dev + 3 * ng, g,
                                                                          reinterpret_cast<float4*>(h->F), h->Nu, h->mask);
        TDLB_CCK(cudaGetLastError());
        TDLB_CCK(cudaStreamSynchronize(h->stream));
        h->cfg = c;
        h->cp = tdlb::make_collide_params(c.nu, c.cs0, c.g3);
        tdlb::set_rest(h->cp, c.initialRho);
        h->cur = 0;
        h->pass = 0;
        h->even = even;
        h->holds_moments = true;
        h->initialised = true;
    });
}

}  // extern "C"
