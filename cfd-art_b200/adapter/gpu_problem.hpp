// GpuProblem: cfd-art's problem_base (headers/problem_base.hpp:18-40) backed
// by the cfdgpu library, for the reference's own, unmodified time loop.
//
// The reference drives a problem through simulation::run_simulation
// (headers/simulation.hpp:36-67) and the splitting scheme named in the
// settings file (headers/splitting_scheme.hpp:29-143).  Registered in place
// of the CPU problem, this class keeps that loop, the settings file, the
// reference's set_ICs and its output writers, and moves the state and the
// time step to the GPU:
//
//   set_ICs     reference set_ICs on the host, then cfd_create (first call)
//               and cfd_upload of the ghosted grid
//   compute_dt  cfd_compute_dt on the device state; the masses it reduces
//               go into the reference problem's mass records, which its
//               masschange writer prints at the end
//   pre_sweep, update_row, update_col
//               nothing: the device fills ghosts and sweeps whole grids
//   post_sweep  the first one after compute_dt runs cfd_step(dt) -- the
//               whole naive or Strang step, as configured -- the others
//               (the splitting scheme's later sweeps of the same step) do
//               nothing
//   output      downloads the state, ghost cells as the reference's grid
//               would hold them, when the reference's output rule is due to
//               write (sourcecode/euler_io.cpp:1235-1261,
//               A/sourcecode/allaire_diffuse_io.cpp:1251-1294), and hands it
//               to the reference's output
//   clone       a handle on the same device solver (the splitting scheme
//               clones the problem for every OpenMP thread)
//
// The host grids the loop passes in are not read or written after set_ICs:
// the state lives on the device.  The loop must call compute_dt before each
// advance_timestep (simulation.hpp:52-54 does).  Errors throw
// std::runtime_error with the library's message; there is no CPU fallback.
//
// CpuProblem is the reference's problem class (Euler, allaire_diffuse) or a
// subclass of it that adds
//     void record_mass(double t, double mass1, double mass2);
// appending to the class's mass records (its compute_dt does this on the CPU).
// Include the reference's headers of the matching tree before this file.
#ifndef CFDGPU_ADAPTER_GPU_PROBLEM_HPP
#define CFDGPU_ADAPTER_GPU_PROBLEM_HPP

#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "cfdgpu.h"
#include "cfdgpu_host.h"

namespace cfdgpu_adapter {

inline void check(int rc, const char* what) {
    if (rc != CFD_OK) {
        char msg[512];
        msg[0] = '\0';
        cfd_last_error(msg, sizeof msg);
        throw std::runtime_error(std::string("[cfdgpu] ") + what + " failed (" +
                                 std::to_string(rc) + "): " + msg);
    }
}

inline void copy_field(char* dst, size_t cap, const std::string& s) {
    std::strncpy(dst, s.c_str(), cap - 1);
    dst[cap - 1] = '\0';
}

// gridtype (headers/typedefs.hpp:19-21: rows of Eigen vectors, ghosts
// included) <-> the library's ghosted AoS layout.
template <class Grid>
void flatten(const Grid& g, int nv, std::vector<double>& out) {
    out.clear();
    for (const auto& row : g)
        for (const auto& U : row)
            for (int k = 0; k < nv; ++k) out.push_back(U(k));
}

template <class Grid>
void unflatten(const std::vector<double>& in, int nv, Grid& g) {
    size_t p = 0;
    for (auto& row : g)
        for (auto& U : row)
            for (int k = 0; k < nv; ++k) U(k) = in[p++];
}

// When the reference's output() writes: the first and last call, every
// T/output_freq of simulated time after the last periodic write, and (Allaire)
// the fixed schlieren times of A/sourcecode/allaire_diffuse_io.cpp:1259.
// Its state advances exactly as output()'s function-static state does.
class OutputRule {
  public:
    OutputRule(double T, int output_freq, bool allaire_frames) : T_(T), freq_(output_freq) {
        if (allaire_frames)
            frames_ = {0.000115, 0.000175, 0.000247, 0.000307, 0.000378, 0.000402, 0.000477,
                       0.001080};
    }
    bool due(int n, double t) {
        bool w = false;
        if (!frames_.empty() && t > frames_[0]) {
            frames_.erase(frames_.begin());
            w = true;
        }
        if (n == 0 || t == T_) return true;
        if (freq_ != 0 && t - last_ > T_ / freq_) {
            last_ = t;
            return true;
        }
        return w;
    }

  private:
    double T_;
    int freq_;
    double last_ = 0.0;
    std::vector<double> frames_;
};

}  // namespace cfdgpu_adapter

template <class CpuProblem, int MODEL>
class GpuProblem : public problem_base {
    struct Device {
        cfd_solver* solver = nullptr;
        cfd_config cfg;
        int nv = 0;
        std::shared_ptr<gridtype> host;  // handed to the reference's output
        std::vector<double> flat;
        std::unique_ptr<cfdgpu_adapter::OutputRule> rule;
        bool every_output = false;
        double dt = 0.0;
        bool step_pending = false;
        int sweeps_left = 0;  // post_sweep calls still due from the step taken
        ~Device() {
            if (solver) cfd_destroy(solver);
        }
    };
    std::shared_ptr<CpuProblem> cpu_;
    std::shared_ptr<Device> dev_;

  public:
    GpuProblem() : cpu_(std::make_shared<CpuProblem>()), dev_(std::make_shared<Device>()) {}

    // Download before every output() call instead of only when the
    // reference's output rule is due (for an output() whose rule differs).
    void set_download_every_output(bool on) { dev_->every_output = on; }

    cfd_solver* solver() const { return dev_->solver; }

    std::shared_ptr<gridtype> set_ICs(settings_file SF, sim_info& params) override {
        using cfdgpu_adapter::check;
        std::shared_ptr<gridtype> g = cpu_->set_ICs(SF, params);
        Device& d = *dev_;
        if (!d.solver) {
            cfd_settings s;
            std::memset(&s, 0, sizeof s);
            s.Nx = SF.Nx;
            s.Ny = SF.Ny;
            s.CFL = SF.CFL;
            s.output_freq = SF.output_freq;
            cfdgpu_adapter::copy_field(s.splitting_scheme, sizeof s.splitting_scheme,
                                       SF.splitting_scheme);
            cfdgpu_adapter::copy_field(s.test_case, sizeof s.test_case, SF.test_case);
            cfdgpu_adapter::copy_field(s.flux_solver, sizeof s.flux_solver, SF.flux_solver);
            cfdgpu_adapter::copy_field(s.riemann_solver, sizeof s.riemann_solver,
                                       SF.riemann_solver);
            cfdgpu_adapter::copy_field(s.problem, sizeof s.problem,
                                       MODEL == CFD_MODEL_ALLAIRE ? "allaire" : "euler");
            check(cfd_settings_config(&s, &d.cfg), "cfd_settings_config");
            // The reference's set_parameters has just filled params: both
            // sides must describe the same grid and time loop.
            const int g_layers = d.cfg.flux_solver == CFD_FLUX_GODUNOV ? 1 : 2;
            if (d.cfg.nx != params.Nx || d.cfg.ny != params.Ny || d.cfg.dx != params.dx ||
                d.cfg.dy != params.dy || d.cfg.T != params.T || d.cfg.cfl != params.CFL ||
                g_layers != params.numGC)
                throw std::runtime_error("[cfdgpu] the library's configuration of test case '" +
                                         SF.test_case + "' differs from the reference's sim_info");
            check(cfd_create(&d.cfg, &d.solver), "cfd_create");
            check(cfd_set_reference_ghosts(d.solver, 1), "cfd_set_reference_ghosts");
            d.nv = cfd_nvar(d.cfg.model);
            d.rule.reset(new cfdgpu_adapter::OutputRule(params.T, params.output_freq,
                                                        MODEL == CFD_MODEL_ALLAIRE));
        }
        // run_simulation calls set_ICs twice (grid, future_grid); both
        // uploads are the same initial state at n = 0, t = 0.
        cfdgpu_adapter::flatten(*g, d.nv, d.flat);
        check(cfd_upload(d.solver, d.flat.data(), CFD_LAYOUT_GHOSTED_AOS, 0, 0.0), "cfd_upload");
        d.host = std::make_shared<gridtype>(*g);
        return g;
    }

    void output(const gridtype&, const sim_info& params, int n, double t) override {
        Device& d = *dev_;
        bool due = d.rule->due(n, t);
        if (due || d.every_output) {
            cfdgpu_adapter::check(
                cfd_download(d.solver, d.flat.data(), CFD_LAYOUT_GHOSTED_AOS_AS_REFERENCE),
                "cfd_download");
            cfdgpu_adapter::unflatten(d.flat, d.nv, *d.host);
        }
        cpu_->output(*d.host, params, n, t);
    }

    double compute_dt(const gridtype&, const sim_info&, int n, double t) override {
        Device& d = *dev_;
        double dt = 0.0;
        cfdgpu_adapter::check(cfd_compute_dt(d.solver, n, t, &dt), "cfd_compute_dt");
        cfd_status st;
        cfdgpu_adapter::check(cfd_get_status(d.solver, &st), "cfd_get_status");
        cpu_->record_mass(t, st.mass1, st.mass2);
        d.dt = dt;
        d.step_pending = true;
        return dt;
    }

    void pre_sweep(gridtype&, const sim_info&) override {}

    void update_row(const gridtype&, gridtype&, const sim_info&, int, double, double) override {}

    void update_col(const gridtype&, gridtype&, const sim_info&, int, double, double) override {}

    void post_sweep(gridtype&, gridtype&, const sim_info&) override {
        Device& d = *dev_;
        if (d.step_pending) {
            d.step_pending = false;
            cfdgpu_adapter::check(cfd_step(d.solver, d.dt), "cfd_step");
            // naive_splitting ends two sweeps with post_sweep, strang_splitting three
            d.sweeps_left = d.cfg.splitting == CFD_SPLIT_STRANG ? 2 : 1;
            return;
        }
        if (d.sweeps_left > 0) {
            --d.sweeps_left;  // a later sweep of the step already taken on the device
            return;
        }
        throw std::runtime_error("[cfdgpu] a time step began without compute_dt; the adapter "
                                 "takes dt from the compute_dt call that precedes each step");
    }

    std::shared_ptr<problem_base> clone() override {
        return std::make_shared<GpuProblem>(*this);
    }
};

#endif
