// tdlb_compute_unit_arch_b200.hpp -- the B200 architecture of tdLBCpp's
// ComputeUnit: a partial specialisation of the reference's
// ComputeUnitArchitecture (tdlbcpp/src/ComputeUnit.h:282-292) that forwards
// every ComputeUnitBase virtual (ComputeUnit.h:86-201) to the C ABI of
// tdlb_b200.h.
//
// Use: include it after the reference's "ComputeUnit.h" (tdlbcpp/src and
// this directory on the include path, link libtdlb_b200.so) and name B200
// where main.cpp's selection (main.cpp:241-256) names CPU or GPU:
//
//     lb = new ComputeUnit<float, QLen::D3Q19, MemoryLayoutIJKL, EgglesSomers, Simple, B200>(cu, flow, outputTree);
//
// Then main.cpp's sequence runs unchanged through the ComputeUnitBase
// pointer: initialise (:261), forcing (:305), and per step collision,
// bounceBackBoundary, streamingPush, moments, forcing (:438-454), plus the
// output calls (setOutputExcludePoints, calcVorticityXY/XZ,
// unsetOutputExcludePoints, :462-496).
//
// B200 is a value outside the reference's enum Architecture {CPU, GPU,
// GPU_MEM_SHARED} (Header.h:39). An unscoped enum without a fixed underlying
// type whose enumerators span 0..2 holds every value 0..3, so the cast is a
// valid constant and the reference's headers need no edit.
//
// The base is built with allocateMemory = false: the lattice lives on the
// GPU behind the handle, and the base's host arrays (Q, F, Nu, O,
// ExcludeOutputPoints) stay NULL. Consequences for callers:
//   * checkpoint_read / checkpoint_write are non-virtual in ComputeUnit.h
//     (:133-134); this class hides them with versions that go through the
//     library. main.cpp calls them through the base pointer (:263, :511), so
//     a build that checkpoints declares those two base functions virtual (a
//     one-word change per line) -- as the reference's own GPU class needs
//     for checkpoint_read (ComputeUnitGpu.h:62);
//   * streamingPull (test-only in the reference) throws: the step streams
//     by pulling inside collision();
//   * errors throw std::runtime_error with the library's message, where the
//     reference's GPU path calls exit() (checkCudaErrors).
// Supported: T = float, 18 populations, EgglesSomers collision, Simple or
// Esotwist streaming, ghost width 1 (main.cpp:225).
#pragma once

#include <cmath>
#include <cstdio>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

#include "ComputeUnit.h"
#include "tdlb_b200.h"

constexpr Architecture B200 = static_cast<Architecture>(GPU_MEM_SHARED + 1);

template <typename T, int QVecSize, MemoryLayoutType MemoryLayout, Collision collisionType, Streaming streamingType>
class ComputeUnitArchitecture<T, QVecSize, MemoryLayout, collisionType, streamingType, B200>
    : public ComputeUnitBase<T, QVecSize, MemoryLayout> {
    static_assert(std::is_same<T, float>::value, "the B200 step computes and stores in FP32 (T = float)");
    static_assert(QVecSize == 18, "the B200 step has 18 moving populations (QLen::D3Q19)");
    static_assert(collisionType == EgglesSomers, "the B200 step implements the EgglesSomers collision");
    static_assert(streamingType == Simple || streamingType == Esotwist, "Simple or Esotwist streaming");

public:
    using Base = ComputeUnitBase<T, QVecSize, MemoryLayout>;

    ComputeUnitArchitecture(ComputeUnitParams cuParams, FlowParams<T> flow, DiskOutputTree outputTree)
        : Base(cuParams, flow, outputTree, /*allocateMemory=*/false) {
        if (this->ghost != 1) throw std::runtime_error("B200 ComputeUnit: ghost (GridParams.multiStep) must be 1");
        tdlb_config c{};
        c.x = (int64_t)this->x;
        c.y = (int64_t)this->y;
        c.z = (int64_t)this->z;
        c.streaming = streamingType == Simple ? TDLB_STREAMING_SIMPLE : TDLB_STREAMING_ESOTWIST;
        c.storage = TDLB_STORAGE_FP32;
        c.initialRho = this->flow.initialRho;
        c.nu = this->flow.nu;
        c.cs0 = this->flow.cs0;
        c.g3 = this->flow.g3;
        c.alpha = this->flow.alpha;
        c.beta = this->flow.beta;
        c.useLES = this->flow.useLES ? 1 : 0;
        const int device = cuParams.deviceID < 0 ? 0 : cuParams.deviceID;
        if (tdlb_create_config(&c, device, &h_) != TDLB_OK)
            throw std::runtime_error(std::string("B200 ComputeUnit: ") + tdlb_last_error(nullptr));
    }
    ComputeUnitArchitecture(const ComputeUnitArchitecture&) = delete;
    ComputeUnitArchitecture& operator=(const ComputeUnitArchitecture&) = delete;
    ~ComputeUnitArchitecture() override {
        if (h_) tdlb_destroy(h_);
    }

    // ---- the time step (ComputeUnit.h:108-201) ----
    void initialise(T rho) override {
        ok(tdlb_initialise(h_, (float)rho));
        this->evenStep = true;
    }
    // One fused launch: streaming of the previous step's populations,
    // moments and collision.
    void collision() override { ok(tdlb_collision(h_)); }
    // The wall rule and the streaming run inside collision(); these keep
    // main.cpp's sequence and the base's evenStep (Esotwist) in step.
    void bounceBackBoundary() override { ok(tdlb_bounce_back(h_)); }
    void streamingPush() override {
        ok(tdlb_streaming_push(h_));
        int even = 1;
        ok(tdlb_get_even_step(h_, &even));
        this->evenStep = even != 0;
    }
    void streamingPull() override {
        throw std::runtime_error("B200 ComputeUnit: streamingPull is not provided (collision() streams by pulling)");
    }
    void moments() override { ok(tdlb_moments(h_)); }

    void forcing(std::vector<PosPolar<tNi, T>>& geom, T alfa, T beta) override {
        to_markers(geom);
        ok(tdlb_forcing(h_, markers_.data(), markers_.size(), (float)alfa, (float)beta));
    }

    // ---- output (ComputeUnitOutput.hpp:20-285) ----
    void setOutputExcludePoints(std::vector<Pos3d<tNi>> geomPoints) override { exclude3d(geomPoints, 1); }
    void setOutputExcludePoints(std::vector<PosPolar<tNi, T>> geomPoints) override {
        to_markers(geomPoints);
        ok(tdlb_set_output_exclude(h_, markers_.data(), markers_.size(), 1));
    }
    void unsetOutputExcludePoints(std::vector<Pos3d<tNi>> geomPoints) override { exclude3d(geomPoints, 0); }
    void unsetOutputExcludePoints(std::vector<PosPolar<tNi, T>> geomPoints) override {
        to_markers(geomPoints);
        ok(tdlb_set_output_exclude(h_, markers_.data(), markers_.size(), 0));
    }

    // The slice j (counted with the ghost layer, as main.cpp passes cutAt)
    // of log |curl u|^2 computed on the device, scaled to 0..255 between its
    // finite minimum and maximum and written as the reference writes it:
    // <formatXZPlaneDir(step, j)>.jpeg through the reference's TooJpeg.
    void calcVorticityXZ(tNi j, RunningParams runParam, int jpegCompression) override {
        (void)jpegCompression;   // the reference writes quality 100 regardless
        const tNi nx = this->x, nz = this->z;
        std::vector<float> v((size_t)nx * nz);
        ok(tdlb_vorticity_xz(h_, (int64_t)(j - this->ghost), v.data()));
        // out[i*z + k]: the reference's picture index zg1*(i-1) + (k-1)
        write_picture(v, (unsigned short)nx, (unsigned short)nz, this->outputTree.formatXZPlaneDir(runParam.step, j));
    }
    void calcVorticityXY(tNi k, RunningParams runParam, int jpegCompression) override {
        (void)jpegCompression;
        const tNi nx = this->x, ny = this->y;
        std::vector<float> v((size_t)nx * ny);
        ok(tdlb_vorticity_xy(h_, (int64_t)(k - this->ghost), v.data()));
        // out[j*x + i]: the reference's picture index (i-1) + xg1*(j-1)
        write_picture(v, (unsigned short)nx, (unsigned short)ny, this->outputTree.formatXYPlaneDir(runParam.step, k));
    }

    // The moments of the cells in the given (ghost-counted) box, as the
    // reference's printDebug prints its Q.
    void printDebug(int fi, int ti, int fj, int tj, int fk, int tk) override {
        std::vector<float> m((size_t)this->x * this->y * this->z * 18);
        ok(tdlb_read_moments(h_, m.data()));
        for (int i = fi; i <= ti; i++)
            for (int j = fj; j <= tj; j++)
                for (int k = fk; k <= tk; k++) {
                    if (i < 1 || j < 1 || k < 1 || i > this->x || j > this->y || k > this->z) continue;
                    const size_t c = (((size_t)(i - 1) * this->y + (j - 1)) * this->z + (k - 1)) * 18;
                    std::printf("index(%d, %d, %d):\n", i, j, k);
                    for (int l = 0; l < 18; l++) std::printf("Q[%d] = %f, ", l, m[c + l]);
                    std::printf("\n");
                }
    }

    // ComputeUnit.hpp:258-316: doubles x, y, z on the device; every new cell
    // takes the moments and Nu of its parent cell.
    void doubleResolutionFullCU() override {
        ok(tdlb_double_resolution(h_));
        const tNi factor = 2;
        this->resolution += factor;
        this->x *= factor;
        this->y *= factor;
        this->z *= factor;
        this->initGridParams();
        this->size = size_t(this->xg) * this->yg * this->zg;
    }

    // ---- checkpoint (ComputeUnit.hpp:318-439), hiding the base's ----
    // Writes the reference's files into the directory the reference would
    // use (DiskOutputTree::getCheckpointDirName), with the AllParams JSON
    // the reference's own writer produces plus the Esotwist parity.
    void checkpoint_write(std::string unit_name, RunningParams run) {
        const std::string dirname = this->outputTree.getCheckpointDirName(run);
        BinFileParams binFormat;    // the reference's checkpoint record (ComputeUnit.hpp:394-403)
        binFormat.filePath = this->outputTree.getAllParamsFilePath(dirname, unit_name);
        binFormat.structName = "checkpoint";
        binFormat.binFileSizeInStructs = static_cast<uint64_t>(this->size);
        binFormat.coordsType = "none";
        binFormat.hasGridtCoords = 0;
        binFormat.hasColRowtCoords = 0;
        binFormat.QDataType = "none";
        binFormat.QOutputLength = QVecSize;
        this->outputTree.setRunningParams(run);
        const nlohmann::json params = this->outputTree.getJsonParams(binFormat, run);
        ok(tdlb_checkpoint_write(h_, dirname.c_str(), unit_name.c_str(), params.dump().c_str()));
    }
    void checkpoint_read(std::string dirname, std::string unit_name) {
        ok(tdlb_checkpoint_read(h_, dirname.c_str(), unit_name.c_str()));
        int even = 1;
        ok(tdlb_get_even_step(h_, &even));
        this->evenStep = even != 0;
    }

    // ---- access to the device lattice (interior cells, (i, j, k) order) ----
    tdlb_handle handle() const { return h_; }
    void read_velocity_density(std::vector<float>& rho, std::vector<float>& ux, std::vector<float>& uy,
                               std::vector<float>& uz) {
        const size_t n = (size_t)this->x * this->y * this->z;
        rho.resize(n);
        ux.resize(n);
        uy.resize(n);
        uz.resize(n);
        ok(tdlb_read_velocity_density(h_, rho.data(), ux.data(), uy.data(), uz.data()));
    }
    void read_force(std::vector<float>& f3) {
        f3.resize((size_t)this->x * this->y * this->z * 3);
        ok(tdlb_read_force(h_, f3.data()));
    }
    void read_nu(std::vector<float>& nu) {
        nu.resize((size_t)this->x * this->y * this->z);
        ok(tdlb_read_nu(h_, nu.data()));
    }

private:
    void ok(int rc) {
        if (rc != TDLB_OK) throw std::runtime_error(std::string("B200 ComputeUnit: ") + tdlb_last_error(h_));
    }

    template <typename P>
    void to_markers(const std::vector<P>& geom) {
        markers_.resize(geom.size());
        for (size_t q = 0; q < geom.size(); q++) {
            tdlb_marker& m = markers_[q];
            m.i = (int64_t)geom[q].i;
            m.j = (int64_t)geom[q].j;
            m.k = (int64_t)geom[q].k;
            m.iCartFraction = (float)geom[q].iCartFraction;
            m.kCartFraction = (float)geom[q].kCartFraction;
            m.uDelta = (float)geom[q].uDelta;
            m.vDelta = (float)geom[q].vDelta;
            m.wDelta = (float)geom[q].wDelta;
            m.pad = 0.f;
        }
    }

    void exclude3d(const std::vector<Pos3d<tNi>>& pts, int on) {
        markers_.assign(pts.size(), tdlb_marker{});
        for (size_t q = 0; q < pts.size(); q++) {
            markers_[q].i = (int64_t)pts[q].i;
            markers_[q].j = (int64_t)pts[q].j;
            markers_[q].k = (int64_t)pts[q].k;
        }
        ok(tdlb_set_output_exclude(h_, markers_.data(), markers_.size(), on));
    }

    static void write_picture(const std::vector<float>& v, unsigned short w, unsigned short h, const std::string& dir) {
        bool have = false;
        float lo = 0.f, hi = 0.f;
        for (float a : v) {
            if (!std::isfinite(a)) continue;
            if (!have || a < lo) lo = a;
            if (!have || a > hi) hi = a;
            have = true;
        }
        std::vector<unsigned char> pict(v.size(), 0);
        const float span = hi > lo ? hi - lo : 1.f;
        for (size_t c = 0; c < v.size(); c++)
            pict[c] = std::isfinite(v[c]) ? (unsigned char)std::floor(255.f * ((v[c] - lo) / span)) : 0;
        TooJpeg::openJpeg(dir + ".jpeg");
        TooJpeg::writeJpeg(pict.data(), w, h, false, 100, false, "Debug");
        TooJpeg::closeJpeg();
    }

    tdlb_handle h_ = nullptr;
    std::vector<tdlb_marker> markers_;
};
