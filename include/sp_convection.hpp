// sp_convection.hpp -- C++ facade with the reference's class names over the C ABI.
//
// Drop-in shapes for drivers written against andyspiros/StencilParareal:
//   ConvectionField         src/Convection/Convection.h:13-20 (device field, 2-cell halo)
//   Convection              src/Convection/Convection.h:22-108
//   RuntimeConfiguration    src/Parareal/RuntimeConfiguration.{h,cpp}
//   Parareal<Prop, Field>   src/Parareal/Parareal.h:38-289
// Differences: errors throw sp::Error (the reference aborts), the number of
// time slices is a configuration value (all slices run on one GPU instead of
// one MPI rank each), and fields are filled through fill()/download() instead
// of STELLA's host/device mirrors.  Header-only; link libstencilparareal.so
// and the CUDA runtime (fields are allocated with cudaMalloc).
#ifndef SP_CONVECTION_HPP_
#define SP_CONVECTION_HPP_

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "sp_abi.h"

namespace sp {

struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

inline void check(int rc, const char* what) {
    if (rc != SP_OK) throw Error(rc, std::string(what) + ": " + sp_last_error());
}

// A device field of FP64 values with the library's halo layout.
class ConvectionField {
public:
    ConvectionField() = default;
    ConvectionField(const ConvectionField&) = delete;
    ConvectionField& operator=(const ConvectionField&) = delete;
    ~ConvectionField() { release(); }

    // DataFieldCUDA::Init(name, domain, kboundary) of the reference.
    void Init(const std::string& name, int isize, int jsize, int ksize) {
        release();
        name_ = name;
        check(sp_field_layout(isize, jsize, ksize, SP_F64, &lay_), "sp_field_layout");
        // zeroed before return: the library's streams do not order after legacy-stream work
        if (cudaMalloc(&ptr_, lay_.total * sizeof(double)) != cudaSuccess ||
            cudaMemset(ptr_, 0, lay_.total * sizeof(double)) != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess)
            throw Error(SP_ERR_NOMEM, "cudaMalloc of field " + name);
    }
    double* data() { return ptr_; }
    const double* data() const { return ptr_; }
    const sp_layout& layout() const { return lay_; }
    const std::string& name() const { return name_; }
    int isize() const { return lay_.ni; }
    int jsize() const { return lay_.nj; }
    int ksize() const { return lay_.nk; }

private:
    void release() {
        if (ptr_) cudaFree(ptr_);
        ptr_ = nullptr;
    }
    double* ptr_ = nullptr;
    sp_layout lay_{};
    std::string name_;
};

class Convection {
public:
    // Convection::Convection (Convection.h:25)
    Convection(int isize, int jsize, int ksize, double dx, double nu0, double nufreq, double cx, double cy,
               double cz, int device = 0, bool upwind = true) {
        sp_params p{isize, jsize, ksize, dx, nu0, nufreq, cx, cy, cz, upwind ? 1 : 0};
        check(sp_convection_create(&p, device, &h_), "sp_convection_create");
    }
    Convection(const Convection&) = delete;
    Convection& operator=(const Convection&) = delete;
    ~Convection() { sp_convection_destroy(h_); }

    // Convection::DoRK4 / DoEuler / DoRK4Timestep / DoEulerTimestep (Convection.h:44-75)
    void DoRK4(ConvectionField& in, ConvectionField& out, double tStart, double dt, int timesteps) {
        check(sp_do_rk4(h_, in.data(), out.data(), tStart, dt, timesteps), "DoRK4");
    }
    void DoEuler(ConvectionField& in, ConvectionField& out, double tStart, double dt, int timesteps) {
        check(sp_do_euler(h_, in.data(), out.data(), tStart, dt, timesteps), "DoEuler");
    }
    void DoRK4Timestep(ConvectionField& in, ConvectionField& out, double t, double dt) { DoRK4(in, out, t, dt, 1); }
    void DoEulerTimestep(ConvectionField& in, ConvectionField& out, double t, double dt) {
        DoEuler(in, out, t, dt, 1);
    }

    // Host <-> device (fillQ + SynchronizeDevice / SynchronizeHost of the drivers).
    void fill(ConvectionField& f, const std::vector<double>& dense) {
        check(sp_field_import(h_, dense.data(), f.data(), SP_F64, 1), "fill");
        synchronize();
    }
    std::vector<double> download(const ConvectionField& f) {
        std::vector<double> d((size_t)f.isize() * f.jsize() * f.ksize());
        check(sp_field_export(h_, f.data(), d.data(), SP_F64, 1), "download");
        return d;
    }
    void synchronize() { check(sp_convection_synchronize(h_), "synchronize"); }
    void autotune(int batch = 1) { check(sp_autotune(h_, SP_F64, batch), "autotune"); }
    sp_convection* handle() { return h_; }

private:
    sp_convection* h_ = nullptr;
};

// RuntimeConfiguration (RuntimeConfiguration.h:13-123, .cpp:7-152).
class RuntimeConfiguration {
public:
    // Defaults of RuntimeConfiguration.cpp:7-13; options with the reference's
    // names ("--nu0 0.1", "--gridSize 128", "--noasync", "--mode serial", ...).
    RuntimeConfiguration(int timeSlices, int argc = 0, char** argv = nullptr) : timeSlices_(timeSlices) {
        if (timeSlices < 1) throw Error(SP_ERR_INVALID, "timeSlices must be >= 1");
        for (int i = 1; i < argc; ++i) {
            std::string a = argv[i];
            if (a.rfind("--", 0) != 0) continue;
            a = a.substr(2);
            auto val = [&]() -> const char* {
                if (i + 1 >= argc) throw Error(SP_ERR_INVALID, "option --" + a + " needs a value");
                return argv[++i];
            };
            if (a == "nu0") nu0_ = std::atof(val());
            else if (a == "nufreq") nufreq_ = std::atof(val());
            else if (a == "cx") cx_ = std::atof(val());
            else if (a == "cy") cy_ = std::atof(val());
            else if (a == "cz") cz_ = std::atof(val());
            else if (a == "gridSize") gridSize_ = std::atoi(val());
            else if (a == "endTime") endTime_ = std::atof(val());
            else if (a == "timeStepsFine") timeStepsFine_ = std::atoi(val());
            else if (a == "timeStepsCoarse") timeStepsCoarse_ = std::atoi(val());
            else if (a == "kmax") kmax_ = std::atoi(val());
            else if (a == "mat") mat_ = true;
            else if (a == "noasync") async_ = false;
            else if (a == "mode") mode_ = val();
        }
        round();
    }
    double nu0() const { return nu0_; }
    double nufreq() const { return nufreq_; }
    double cx() const { return cx_; }
    double cy() const { return cy_; }
    double cz() const { return cz_; }
    int timeSlices() const { return timeSlices_; }
    int timeStepsFine() const { return timeStepsFine_; }
    int timeStepsCoarse() const { return timeStepsCoarse_; }
    int gridSize() const { return gridSize_; }
    double endTime() const { return endTime_; }
    int kmax() const { return kmax_; }
    bool mat() const { return mat_; }
    bool async() const { return async_; }
    const std::string& mode() const { return mode_; }
    void set_nu0(double x) { nu0_ = x; }
    void set_nufreq(double x) { nufreq_ = x; }
    void set_gridSize(int x) { gridSize_ = x; }
    void set_endTime(double x) { endTime_ = x; }
    void set_timeStepsFine(int x) { timeStepsFine_ = x; round(); }
    void set_timeStepsCoarse(int x) { timeStepsCoarse_ = x; round(); }
    void set_kmax(int x) { kmax_ = x; }
    void set_async(bool x) { async_ = x; }
    double dx() const { return 1. / gridSize_; }
    double dtFine() const { return endTime_ / timeStepsFine_; }
    double dtCoarse() const { return endTime_ / timeStepsCoarse_; }
    int timeStepsFinePerTimeSlice() const { return timeStepsFine_ / timeSlices_; }
    int timeStepsCoarsePerTimeSlice() const { return timeStepsCoarse_ / timeSlices_; }
    double timeSliceSize() const { return endTime_ / timeSlices_; }
    double cflFine() const { return cfl(dtFine()); }
    double cflCoarse() const { return cfl(dtCoarse()); }

private:
    // RuntimeConfiguration.cpp:133-151: totals rounded up to a multiple of the slice count
    void round() {
        if (timeStepsFine_ % timeSlices_ != 0) timeStepsFine_ = (timeStepsFine_ / timeSlices_ + 1) * timeSlices_;
        if (timeStepsCoarse_ % timeSlices_ != 0)
            timeStepsCoarse_ = (timeStepsCoarse_ / timeSlices_ + 1) * timeSlices_;
    }
    double cfl(double dt) const {
        const double c = std::max(std::max(cx_, cy_), cz_);
        const double dt_dx = dt / dx();
        return std::max(1.5 * nu0_ * dt_dx / dx(), c * dt_dx);
    }
    double nu0_ = 1., nufreq_ = 0., cx_ = 1., cy_ = 1., cz_ = 1.;
    int gridSize_ = 32;
    double endTime_ = 0.05;
    int timeSlices_ = 1;
    int timeStepsFine_ = 128, timeStepsCoarse_ = 32;
    int kmax_ = 5;
    bool mat_ = false, async_ = true;
    std::string mode_ = "compare";
};

// Parareal<PropagatorT, FieldType> (Parareal.h:38-289): all slices on one GPU.
// The coarse propagator is the reference's DoEuler in FP64 by default;
// coarse_scheme / coarse_precision / coarse_delta select the other variants.
template <typename PropagatorT, typename FieldType>
class Parareal {
public:
    Parareal(PropagatorT& propagator, FieldType& initial, FieldType& solution, double tStart,
             const RuntimeConfiguration& conf, int coarse_scheme = SP_COARSE_EULER, int coarse_precision = SP_F64,
             int coarse_delta = -1)
        : qinitial_(initial), q_(solution), tStart_(tStart) {
        sp_parareal_cfg c{};
        c.endTime = conf.endTime();
        c.timeSlices = conf.timeSlices();
        c.timeStepsFine = conf.timeStepsFine();
        c.timeStepsCoarse = conf.timeStepsCoarse();
        c.kmax = conf.kmax();
        c.async = conf.async() ? 1 : 0;
        c.coarse_scheme = coarse_scheme;
        c.coarse_precision = coarse_precision;
        c.tol_kind = SP_TOL_NONE;
        c.skip_converged = 1;
        c.coarse_delta = coarse_delta < 0 ? (coarse_precision == SP_F32 ? 1 : 0) : coarse_delta;
        check(sp_parareal_create(propagator.handle(), &c, &h_), "sp_parareal_create");
    }
    Parareal(const Parareal&) = delete;
    Parareal& operator=(const Parareal&) = delete;
    ~Parareal() { sp_parareal_destroy(h_); }

    void DoParallel(const FieldType* reference = nullptr) {
        check(sp_parareal_do_parallel(h_, qinitial_.data(), q_.data(), reference ? reference->data() : nullptr,
                                      &report_),
              "DoParallel");
    }
    // times: [total, fine, coarse] device seconds of DoParallel (the reference
    // records MPI_Wtime stamps per phase and rank, Parareal.h:173-248).
    void DoTimedParallel(std::vector<double>& times) {
        DoParallel();
        times = {report_.seconds, report_.seconds_fine, report_.seconds_coarse};
    }
    void DoSerial() { check(sp_parareal_do_serial(h_, qinitial_.data(), q_.data()), "DoSerial"); }
    const sp_parareal_report& report() const { return report_; }

private:
    FieldType& qinitial_;
    FieldType& q_;
    double tStart_;
    sp_parareal* h_ = nullptr;
    sp_parareal_report report_{};
};

}  // namespace sp

#endif  // SP_CONVECTION_HPP_
