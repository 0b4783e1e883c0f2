// Command-line drop-in for MorphoShell's executable
// (preliminary_setup.cpp:56-71):
//
//   morphoshell_gpu settings.txt mesh.vtk [ansatz.vtk] [--out DIR]
//                   [--max-steps N] [--mixed] [--no-output] [--keep-going]
//
// Runs the set-up on the host and the dynamics loop on the GPU.  Output
// files go to DIR (default: output_using_<settings>_and_<mesh>).
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../../include/morphoshell_host.h"

static std::string stem(const std::string& p) {
    size_t s = p.find_last_of('/');
    std::string f = s == std::string::npos ? p : p.substr(s + 1);
    size_t d = f.find_last_of('.');
    return d == std::string::npos ? f : f.substr(0, d);
}

int main(int argc, char** argv) {
    std::vector<std::string> pos;
    std::string out_dir;
    long long max_steps = 0;
    int mixed = 0, write = 1, keep_going = 0;
    for (int i = 1; i < argc; ++i) {
        std::string a = argv[i];
        if (a == "--out" && i + 1 < argc) out_dir = argv[++i];
        else if (a == "--max-steps" && i + 1 < argc) max_steps = std::atoll(argv[++i]);
        else if (a == "--mixed") mixed = 1;
        else if (a == "--no-output") write = 0;
        else if (a == "--keep-going") keep_going = 1;
        else pos.push_back(a);
    }
    if (pos.size() != 2 && pos.size() != 3) {
        std::fprintf(stderr,
                     "Error: Please provide at least one settings file path followed by one data file path as "
                     "command line arguments.\nA path to a file with ansatz degrees of freedom can be given as a "
                     "third argument if desired.\n");
        return -1;
    }
    if (out_dir.empty()) out_dir = "output_using_" + stem(pos[0]) + "_and_" + stem(pos[1]);
    msh_model* m = nullptr;
    if (msh_load(pos[0].c_str(), pos[1].c_str(), pos.size() == 3 ? pos[2].c_str() : nullptr, 0, &m) != 0) {
        std::fprintf(stderr, "%s\n", msh_last_error());
        return -1;
    }
    msh_run_options o;
    std::memset(&o, 0, sizeof(o));
    o.max_steps = max_steps;
    o.stop_at_final_equilibrium = keep_going ? 0 : 1;
    o.write_outputs = write;
    o.precision = mixed ? MS_PRECISION_MIXED : MS_PRECISION_FP64;
    o.device = -1;
    o.output_dir = out_dir.c_str();
    msh_run_result r;
    int rc = msh_run(m, &o, &r, nullptr);
    msh_free(m);
    if (rc != 0) {
        std::fprintf(stderr, "%s\n", msh_last_error());
        return -1;
    }
    std::printf("steps %lld, dial factor %.6f, %d equilibria, %.3f s\n", (long long)r.steps, r.final_dial_factor,
                r.equilibria_reached, r.wall_seconds);
    return 0;
}
