// tdlb_compute_unit_b200.hpp -- C++ host mirror of tdLBCpp's ComputeUnit
// over the C ABI of include/tdlb_b200.h (header only).
//
// It keeps the reference's per-step call sequence of main.cpp:438-454
//     lb->collision(); lb->bounceBackBoundary(); lb->streamingPush();
//     lb->moments();   lb->forcing(geomFORCING, flow.alpha, flow.beta);
// and the reference's marker vectors: forcing() takes any std::vector of a
// PosPolar-like type with fields i, j, k, iCartFraction, kCartFraction,
// uDelta, vDelta, wDelta (PosPolar<tNi,T>, Forcing.hpp:72-150). Indices are
// the reference's (without ghost), as the reference passes them.
//
// Errors: the reference exits (checkCudaErrors) or throws std::runtime_error
// (params); here every failing call throws std::runtime_error with the
// library's message.
#pragma once

#include <stdexcept>
#include <string>
#include <vector>

#include "tdlb_b200.h"

namespace tdlb {

class ComputeUnitB200 {
public:
    // From the reference's input-file JSON text (main.cpp:135-164).
    ComputeUnitB200(const std::string& inputJson, int device = 0) {
        check_create(tdlb_create(inputJson.c_str(), device, &h_));
        fetch_dims();
    }
    // From an explicit configuration.
    explicit ComputeUnitB200(const tdlb_config& cfg, int device = 0) {
        check_create(tdlb_create_config(&cfg, device, &h_));
        fetch_dims();
    }
    ComputeUnitB200(const ComputeUnitB200&) = delete;
    ComputeUnitB200& operator=(const ComputeUnitB200&) = delete;
    ~ComputeUnitB200() {
        if (h_) tdlb_destroy(h_);
    }

    // ComputeUnitBase virtuals (ComputeUnit.h:110-200)
    void initialise(float rho) { check(tdlb_initialise(h_, rho)); }
    void collision() { check(tdlb_collision(h_)); }
    void bounceBackBoundary() { check(tdlb_bounce_back(h_)); }
    void streamingPush() { check(tdlb_streaming_push(h_)); }
    void moments() { check(tdlb_moments(h_)); }

    template <typename PosPolarT>
    void forcing(const std::vector<PosPolarT>& geom, float alfa, float beta) {
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
        check(tdlb_forcing(h_, markers_.data(), markers_.size(), alfa, beta));
    }

    // Field access (interior cells, (i, j, k) order).
    std::vector<float> moments_aos() {
        std::vector<float> out((size_t)x * y * z * 18);
        check(tdlb_read_moments(h_, out.data()));
        return out;
    }
    void velocity_density(std::vector<float>& rho, std::vector<float>& ux, std::vector<float>& uy,
                          std::vector<float>& uz) {
        const size_t n = (size_t)x * y * z;
        rho.resize(n); ux.resize(n); uy.resize(n); uz.resize(n);
        check(tdlb_read_velocity_density(h_, rho.data(), ux.data(), uy.data(), uz.data()));
    }
    bool evenStep() {
        int e = 1;
        check(tdlb_get_even_step(h_, &e));
        return e != 0;
    }
    void synchronize() { check(tdlb_synchronize(h_)); }
    tdlb_handle handle() const { return h_; }

    // checkpoint_write / checkpoint_read (ComputeUnit.hpp:318-439); the
    // directory is passed in, params_json carries the run's params sections.
    void checkpoint_write(const std::string& dir, const std::string& unit_name, const std::string& params_json = "") {
        check(tdlb_checkpoint_write(h_, dir.c_str(), unit_name.c_str(), params_json.empty() ? nullptr : params_json.c_str()));
    }
    void checkpoint_read(const std::string& dir, const std::string& unit_name) {
        check(tdlb_checkpoint_read(h_, dir.c_str(), unit_name.c_str()));
    }

    int64_t x = 0, y = 0, z = 0;

private:
    void check(int rc) {
        if (rc != TDLB_OK) throw std::runtime_error(std::string("tdlb: ") + tdlb_last_error(h_));
    }
    static void check_create(int rc) {
        if (rc != TDLB_OK) throw std::runtime_error(std::string("tdlb create: ") + tdlb_last_error(nullptr));
    }
    void fetch_dims() { check(tdlb_get_dims(h_, &x, &y, &z)); }

    tdlb_handle h_ = nullptr;
    std::vector<tdlb_marker> markers_;
};

}  // namespace tdlb
