// The reference's own driver program (E/sourcecode/main.cpp:17-48,
// A/sourcecode/main.cpp:18-49) with the GPU problem registered: the settings
// file, the simulation loop (headers/simulation.hpp), the splitting schemes,
// set_ICs and the output writers are the reference's, compiled from its
// sources; only the problem object differs.  Build it against one tree's headers and objects:
//
//   Euler tree:    -I<E>/headers  <E objects>  -lcfdgpu
//   Allaire tree:  -DCFDGPU_ADAPTER_ALLAIRE -I<A>/headers  <A objects>  -lcfdgpu
//
// (oracle/Makefile's `adapter` target does both).  The settings file's
// `problem` key must name the build's model: "euler", or "allaire" for the
// Allaire tree (whose own main registers only its Euler class,
// A/sourcecode/main.cpp:27-36).
#include <cstdio>
#include <exception>
#include <iostream>
#include <memory>
#include <string>

#include "problem_base.hpp"
#include "settings_file.hpp"
#include "simulation.hpp"
#ifdef CFDGPU_ADAPTER_ALLAIRE
#include "allaire_diffuse.hpp"
#else
#include "euler_problem.hpp"
#endif

#include "gpu_problem.hpp"

// The reference problems keep their mass records protected; their compute_dt
// appends to them.  On the GPU path the adapter appends the device's sums.
#ifdef CFDGPU_ADAPTER_ALLAIRE
class AllaireRecords : public allaire_diffuse {
  public:
    void record_mass(double t, double m1, double m2) {
        time.push_back(t);
        mass1.push_back(m1);
        mass2.push_back(m2);
    }
};
using GpuSolverProblem = GpuProblem<AllaireRecords, CFD_MODEL_ALLAIRE>;
static const char* const kProblemKey = "allaire";
#else
class EulerRecords : public Euler {
  public:
    void record_mass(double t, double m1, double) {
        time.push_back(t);
        mass.push_back(m1);
    }
};
using GpuSolverProblem = GpuProblem<EulerRecords, CFD_MODEL_EULER>;
static const char* const kProblemKey = "euler";
#endif

int main(int argc, char* argv[]) {
    if (argc < 2) {
        std::fprintf(stderr, "usage: %s <settingsfile>\n", argv[0]);
        return 2;
    }
    settings_file sf;
    sf.read_settings_file(argv[1]);
    if (sf.problem != kProblemKey) {
        std::fprintf(stderr, "[main] problem '%s' is not registered in this build\n",
                     sf.problem.c_str());
        return 2;
    }
    std::shared_ptr<problem_base> problem = std::make_shared<GpuSolverProblem>();
    simulation sim(sf, problem);
    try {
        int status = sim.run_simulation();
        std::cout << "[main] Simulation exited with status = " << status << std::endl;
        return status;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "%s\n", e.what());
        return 1;
    }
}
