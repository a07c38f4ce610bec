// run-cfd-simulation: drop-in for the reference's run-euler-equations-simulation.
//
//   run-cfd-simulation <settingsfile.txt>
//
// Reads the reference settings file (headers/settings_file.hpp:35-71), builds
// the initial condition with the restated set_ICs hooks, runs the time loop
// of headers/simulation.hpp:48-61 with compute_dt and the split step on the
// GPU, and writes the reference's gnuplot outputs with its cadence
// (sourcecode/euler_io.cpp:1235-1261, A/sourcecode/allaire_diffuse_io.cpp:1251-1294).
// The solver keeps the reference's ghost values, so the outputs that read
// ghost cells (schlieren at the domain edge, Allaire lineouts) are the
// reference's too.
#include <chrono>
#include <cmath>
#include <cstdio>
#include <string>
#include <vector>

#include "cfdgpu.h"
#include "cfdgpu_host.h"

static int die(const char* what, int rc) {
    char msg[512];
    cfd_last_error(msg, sizeof msg);
    std::fprintf(stderr, "[run-cfd-simulation] %s failed (%d): %s\n", what, rc, msg);
    return 1;
}

int main(int argc, char** argv) {
    if (argc < 2) {
        std::fprintf(stderr, "usage: %s <settingsfile>\n", argv[0]);
        return 2;
    }
    cfd_settings sf;
    int rc = cfd_read_settings(argv[1], &sf);
    if (rc) return die("reading the settings file", rc);
    cfd_config cfg;
    if ((rc = cfd_settings_config(&sf, &cfg))) return die("settings", rc);
    size_t elems = 0;
    cfd_ic_grid_elems(&cfg, &elems);
    std::vector<double> grid(elems);
    if ((rc = cfd_settings_ic(&sf, &cfg, grid.data()))) return die("initial condition", rc);
    cfd_solver* s = nullptr;
    if ((rc = cfd_create(&cfg, &s))) return die("cfd_create", rc);
    if ((rc = cfd_set_reference_ghosts(s, 1))) return die("cfd_set_reference_ghosts", rc);
    if ((rc = cfd_upload(s, grid.data(), CFD_LAYOUT_GHOSTED_AOS, 0, 0.0))) return die("upload", rc);

    const std::string base = sf.basename;
    const double T = cfg.T;
    const double outputinterval = T / sf.output_freq;
    double lastoutputtime = 0.0;
    std::vector<double> tt, m1, m2;
    const bool allaire = cfg.model == CFD_MODEL_ALLAIRE;
    // A/sourcecode/allaire_diffuse_io.cpp:1259: extra schlieren frames
    std::vector<double> schlieren_times;
    if (allaire)
        schlieren_times = {0.000115, 0.000175, 0.000247, 0.000307, 0.000378, 0.000402, 0.000477,
                           0.001080};
    bool have = false;  // grid holds the state of this output call
    // schlieren frames: |grad rho| formed on the device, nx*ny values copied back
    std::vector<double> field((size_t)cfg.nx * cfg.ny);
    auto schlieren = [&](double t) -> int {
        int r = cfd_schlieren(s, CFD_LAYOUT_GHOSTED_AOS_AS_REFERENCE, field.data());
        if (!r) r = cfd_write_schlieren_field(&cfg, field.data(), base.c_str(), t);
        return r;
    };
    auto fetch = [&]() -> int {
        if (have) return 0;
        have = true;
        return cfd_download(s, grid.data(), CFD_LAYOUT_GHOSTED_AOS_AS_REFERENCE);
    };
    auto output = [&](int n, double t) -> int {
        have = false;
        int r;
        if (!schlieren_times.empty() && t > schlieren_times[0]) {
            if ((r = schlieren(t))) return r;
            schlieren_times.erase(schlieren_times.begin());
        }
        bool final_out = (t == T);
        bool due = (n == 0 || final_out) ||
                   (sf.output_freq != 0 && t - lastoutputtime > outputinterval);
        if (!due) return 0;
        if ((r = fetch())) return r;
        cfd_write_state(&cfg, grid.data(), base.c_str(), t);
        if ((r = schlieren(t))) return r;
        if (allaire && (n == 0 || final_out)) cfd_write_lineout(&cfg, grid.data(), base.c_str(), n);
        if (final_out && !tt.empty())
            cfd_write_masschange(&cfg, base.c_str(), (int)tt.size(), tt.data(), m1.data(), m2.data());
        if (!(n == 0 || final_out)) lastoutputtime = t;
        return 0;
    };

    std::printf("[main] Beginning simulation..\n");
    auto t0 = std::chrono::steady_clock::now();
    int n = 0;
    double t = 0.0;
    while (t < T && (sf.steps <= 0 || n < sf.steps)) {
        if ((rc = output(n, t))) return die("output", rc);
        double dt;
        if ((rc = cfd_compute_dt(s, n, t, &dt))) return die("compute_dt", rc);
        cfd_status st;
        cfd_get_status(s, &st);
        tt.push_back(t);
        m1.push_back(st.mass1);
        m2.push_back(st.mass2);
        if ((rc = cfd_step(s, dt))) return die("step", rc);
        t += dt;
        n++;
        if (std::fabs(t - T) < 1e-12) t = T;
    }
    if ((rc = output(n, t))) return die("output", rc);
    cfd_synchronize(s);
    double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    cfd_status st;
    cfd_get_status(s, &st);
    std::printf("[simulation] %d steps, t = %g\n", n, t);
    std::printf("[main] The wall clock runtime was %gs.\n", secs);
    // One machine-readable line: the run's size, time and the device's event counters
    // (wall time includes the initial upload and every output written).
    const double updates = (double)cfg.nx * cfg.ny * n;
    std::printf("[metrics] {\"model\": \"%s\", \"nx\": %d, \"ny\": %d, \"steps\": %d, \"t\": %.17g, "
                "\"cell_updates\": %.17g, \"wall_s\": %.6f, \"gcell_updates_per_s\": %.6g, "
                "\"counters\": {\"unphysical_input\": %llu, \"slope_zeroed\": %llu, "
                "\"first_order\": %llu, \"fixup\": %llu, \"unphysical_output\": %llu}}\n",
                allaire ? "allaire" : "euler", cfg.nx, cfg.ny, n, t, updates, secs,
                secs > 0.0 ? updates / secs / 1e9 : 0.0, st.counters[CFD_CNT_UNPHYSICAL_INPUT],
                st.counters[CFD_CNT_SLOPE_ZEROED], st.counters[CFD_CNT_FIRST_ORDER],
                st.counters[CFD_CNT_FIXUP], st.counters[CFD_CNT_UNPHYSICAL_OUTPUT]);
    if (st.counters[CFD_CNT_UNPHYSICAL_INPUT] || st.counters[CFD_CNT_UNPHYSICAL_OUTPUT])
        std::printf("[main] warning: %llu unphysical states reached the flux solver\n",
                    st.counters[CFD_CNT_UNPHYSICAL_INPUT] + st.counters[CFD_CNT_UNPHYSICAL_OUTPUT]);
    cfd_destroy(s);
    return 0;
}
