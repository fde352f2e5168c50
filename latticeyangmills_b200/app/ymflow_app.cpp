// ymflow_flow — drop-in replacement for the reference's LatticeQCD binary run
// with a FLOW input file (src/MainPrograms/LatticeQCDMain.cpp:5-30), on one B200.
//
//   ymflow_flow input.json
//
// Same JSON keys and validation as the reference's JsonInput layer for FLOW:
//   "App": {"type": "FLOW", "params": {"epsilon": e, "tauFinal": T}}   (jsonapp.cpp:49-64)
//   "LatticeSize"/"SubLatticeSize": {"x","y","z","t"}                   (jsonlattice.cpp:11-73)
//   "Action": {"type": "puregauge", "params": {"beta": b}}              (jsonaction.cpp:60-89)
//   "Observables": [... "superobs" ...]                                 (jsonobservable.cpp:64-78)
//   "InputDir", "OutputDir"                                             (jsondirectories.cpp:20-55)
// Optional keys this driver adds, outside App.params (whose size the reference
// checks): "Precision" ("fp64" default, "fp32_18", "fp32_12"), "ReunitEvery"
// (mixed precisions, default 10), "Device" (default 0), "Endian" ("little"
// default; "big" reads the byte-reversed files of the reference's commented
// "FOR CHROMA" reader, inputconf.cpp:135-143), "IOChunkSites" (sites per
// streamed read, default 65536).
//
// Configurations are streamed: ymflow_load_file reads each file in chunks
// through two pinned buffers, overlapping the reads with the device copies
// (byte reversal on the device), so no whole-field host copy is held (a 64^4
// .bin is 9.7 GB).
//
// Same inputs and outputs: every *.bin in InputDir in sorted order
// (inputconf.cpp:76-82), int(tauFinal/epsilon) rows per configuration with
// int(tauFinal/epsilon) - 1 flow steps and a measurement after each
// (wilsonflow.cpp:115-136), OutputDir/flow/confNNNN.dat with "%lf\t" cells
// (outputobs.cpp:64-84), OutputDir/observables.dat header (outputobs.cpp:30-40),
// and the terminal lines of outputterm.cpp.  Added: OutputDir/flow/confNNNN.full.dat
// with every number at full precision ("%.17g") and t^2<E>.
//
// SubLatticeSize: the reference splits the lattice into sub-lattices, one per
// MPI rank (parallel.cpp:57-100).  When it splits only the time extent (x, y,
// z equal to LatticeSize's, t dividing it), this driver flows each
// configuration as that many time slabs, one per GPU (round-robin over the
// B200s present from "Device"), with the halo exchange inside the stage kernel
// (ymflow_slab_group_flow).  Any other SubLatticeSize is validated and the
// lattice flows whole on one GPU.
#include <sys/stat.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <dirent.h>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "json_lite.h"
#include "ymflow.h"

namespace {

[[noreturn]] void die(const std::string& msg) {
    std::fprintf(stderr, "LatticeQCD Error: %s\n", msg.c_str());
    std::exit(1);
}

struct Input {
    double epsilon = 0.0, tau_final = 0.0, beta = 0.0;
    int size[4] = {0, 0, 0, 0};
    int sub[4] = {0, 0, 0, 0};
    std::string input_dir, output_dir;
    int precision = YMFLOW_FP64;
    int reunit_every = 10;
    int device = 0;
    bool big_endian = false;
    int64_t chunk_sites = 65536;
};

void read_extents(const jl::Value& root, const char* key, int out[4]) {
    if (root.count(key) == 0) die(std::string("no ") + key + " specified");
    const jl::Value& v = root[key];
    if (v.size() != 4 || v["x"].size() != 1 || v["y"].size() != 1 || v["z"].size() != 1 || v["t"].size() != 1)
        die(std::string("wrong ") + key + " specification\nCorrect format is:\n \"" + key +
            "\" : {\n   \"x\" : Nx, \n   \"y\" : Ny, \n   \"z\" : Nz, \n   \"t\" : Nt  \n}");
    const char* names[4] = {"x", "y", "z", "t"};
    for (int i = 0; i < 4; i++) {
        if (v[names[i]].kind != jl::Value::Number) die(std::string(key) + " extents must be numbers");
        out[i] = int(v[names[i]].num);
        if (out[i] < 1) die(std::string(key) + " extents must be >= 1");
    }
}

Input parse_input(const char* path) {
    std::ifstream f(path);
    if (!f) die(std::string("cannot open input file ") + path);
    std::stringstream ss;
    ss << f.rdbuf();
    jl::Value root;
    try {
        root = jl::Parser(ss.str()).parse();
    } catch (const std::exception& e) {
        die(e.what());
    }
    Input in;
    // App (jsonapp.cpp:11-64)
    const jl::Value& app = root["App"];
    if (app["type"].size() == 0) die("no App specified");
    if (app["type"].size() != 1) die("wrong App specification");
    if (!app["type"].is_string("FLOW")) {
        if (app["type"].is_string("GFR") || app["type"].is_string("PGFG"))
            die("App \"" + app["type"].str + "\" is not part of this drop-in; only \"FLOW\" is provided");
        die("unknown App " + (app["type"].kind == jl::Value::String ? app["type"].str : std::string("?")));
    }
    const jl::Value& params = app["params"];
    if (params.size() != 2 || params["epsilon"].size() != 1 || params["tauFinal"].size() != 1)
        die("wrong \"FLOW\" app specification\nCorrect format:\"App\" : {\n   \"type\" : \"FLOW\", \n"
            "   \"params\" : { \n       \"epsilon\" : epsilon, \n       \"tauFinal\" : tauFinal \n   }\n}");
    in.epsilon = params["epsilon"].num;
    in.tau_final = params["tauFinal"].num;
    // lattice (jsonlattice.cpp:11-73)
    read_extents(root, "LatticeSize", in.size);
    read_extents(root, "SubLatticeSize", in.sub);
    // action (jsonaction.cpp:12-89)
    if (root.count("Action") == 0) die("no Action specified");
    const jl::Value& act = root["Action"];
    if (act["type"].size() != 1 || act["params"].size() == 0) die("wrong Action specification");
    if (!act["type"].is_string("puregauge")) die("unknown Action");
    if (act["params"].size() != 1 || act["params"]["beta"].size() != 1)
        die("wrong \"puregauge\" action specification");
    in.beta = act["params"]["beta"].num;
    // observables (jsonobservable.cpp:12-78)
    if (root.count("Observables") == 0 || root["Observables"].size() == 0) die("no Observables specified");
    bool superobs = false;
    for (const jl::Value& o : root["Observables"].arr) {
        const std::string s = o.kind == jl::Value::String ? o.str : std::string();
        if (s != "plaquette" && s != "energydensity" && s != "topologicalcharge" && s != "superobs")
            die("unknown Observable \"" + s + "\"");
        superobs = superobs || s == "superobs";
    }
    if (!superobs) die("FLOW measures through \"superobs\"; add it to Observables");
    // directories (jsondirectories.cpp:20-55)
    if (root.count("InputDir") == 0) die("no InputDir specified");
    if (root.count("OutputDir") == 0) die("no OutputDir specified");
    in.input_dir = root["InputDir"].str;
    in.output_dir = root["OutputDir"].str;
    // additions
    if (root.count("Precision")) {
        const std::string p = root["Precision"].str;
        if (p == "fp64") in.precision = YMFLOW_FP64;
        else if (p == "fp32_18") in.precision = YMFLOW_FP32_18;
        else if (p == "fp32_12") in.precision = YMFLOW_FP32_12;
        else die("unknown Precision \"" + p + "\" (fp64, fp32_18, fp32_12)");
    }
    if (root.count("ReunitEvery")) in.reunit_every = int(root["ReunitEvery"].num);
    if (root.count("Device")) in.device = int(root["Device"].num);
    if (root.count("Endian")) {
        const std::string e = root["Endian"].str;
        if (e == "big") in.big_endian = true;
        else if (e != "little") die("unknown Endian \"" + e + "\" (little, big)");
    }
    if (root.count("IOChunkSites")) {
        in.chunk_sites = int64_t(root["IOChunkSites"].num);
        if (in.chunk_sites < 1) die("IOChunkSites must be >= 1");
    }
    if (!(in.epsilon > 0.0) || !(in.tau_final >= 0.0)) die("epsilon must be > 0 and tauFinal >= 0");
    return in;
}

std::vector<std::string> input_list(const std::string& dir) {
    std::vector<std::string> out;
    DIR* d = opendir(dir.c_str());
    if (!d) die("cannot open InputDir " + dir);
    while (dirent* e = readdir(d)) {
        std::string n = e->d_name;
        if (n.size() > 4 && n.compare(n.size() - 4, 4, ".bin") == 0) out.push_back(dir + "/" + n);
    }
    closedir(d);
    std::sort(out.begin(), out.end());
    return out;
}

void check(int st, ymflow_ctx* ctx, const char* what) {
    if (st != YMFLOW_OK) die(std::string(what) + ": " + ymflow_last_error(ctx) + " (status " + std::to_string(st) + ")");
}

}  // namespace

int main(int argc, char** argv) {
    const auto start = std::chrono::system_clock::now();
    if (argc != 2) die("wrong numper of command line arguments provided.");
    const Input in = parse_input(argv[1]);

    std::printf("Total Lattice Size: %2i %2i %2i %2i\n", in.size[0], in.size[1], in.size[2], in.size[3]);
    std::printf("Sublattice Size:    %2i %2i %2i %2i\n\n", in.sub[0], in.sub[1], in.sub[2], in.sub[3]);
    // time slabs when SubLatticeSize splits only t
    int nslabs = 1;
    if (in.sub[0] == in.size[0] && in.sub[1] == in.size[1] && in.sub[2] == in.size[2] && in.sub[3] < in.size[3] &&
        in.size[3] % in.sub[3] == 0) {
        if ((int64_t(in.size[0]) * in.size[1] * in.size[2]) % 32 == 0)
            nslabs = in.size[3] / in.sub[3];
        else
            std::fprintf(stderr, "ymflow: time slabs need x y z divisible by 32; flowing the lattice whole\n");
    }
    std::printf("Number of Processors: \t\t%i\n", nslabs);
    std::printf("Number of Active Processors: \t%i\n\n", nslabs);

    mkdir(in.output_dir.c_str(), 0755);
    mkdir((in.output_dir + "/flow").c_str(), 0755);
    if (FILE* o = std::fopen((in.output_dir + "/observables.dat").c_str(), "w+")) {
        std::fprintf(o, "Step\t");
        std::fprintf(o, "%s\t", "SuperObs");
        std::fprintf(o, "\n");
        std::fclose(o);
    }

    int st = 0;
    std::vector<ymflow_ctx*> slabs;  // one context per slab (one slab: the whole lattice)
    if (nslabs == 1) {
        ymflow_ctx* ctx = ymflow_create(in.size, in.precision, in.device, &st);
        if (!ctx) die(std::string("ymflow_create: ") + ymflow_last_error(nullptr));
        slabs.push_back(ctx);
    } else {
        int ndev = 0;
        ymflow_device_count(&ndev);
        for (int i = 0; i < nslabs; i++) {
            const int dev = ndev > 0 ? (in.device + i) % ndev : in.device;
            ymflow_ctx* c = ymflow_create_slab(in.size, i * in.sub[3], in.sub[3], in.precision, dev, &st);
            if (!c) die(std::string("ymflow_create_slab: ") + ymflow_last_error(nullptr));
            slabs.push_back(c);
        }
    }
    ymflow_ctx* ctx = slabs[0];

    const int rows = int(in.tau_final / in.epsilon);  // wilsonflow.cpp:117
    const int nsteps = rows > 1 ? rows - 1 : 0;
    std::vector<ymflow_obs> obs(size_t(nsteps) + 2);

    int conf_num = 0;
    for (const std::string& path : input_list(in.input_dir)) {
        for (ymflow_ctx* c : slabs)  // each slab reads its own part of the file
            check(ymflow_load_file(c, path.c_str(), in.big_endian ? YMFLOW_IO_BIG_ENDIAN : 0, in.chunk_sites), c,
                  "load");
        int n_out = 0;
        if (nslabs == 1)
            check(ymflow_flow(ctx, in.epsilon, nsteps, 1, in.reunit_every, obs.data(), int(obs.size()), &n_out), ctx,
                  "flow");
        else
            check(ymflow_slab_group_flow(slabs.data(), nslabs, in.epsilon, nsteps, 1, in.reunit_every, obs.data(),
                                         int(obs.size()), &n_out),
                  ctx, "flow");
        // OutputTerm::writeObs (outputterm.cpp:58-66) for the configuration as read
        std::printf("Configuration Number %4i\n", conf_num);
        std::printf("\t%s\t = %g \n", "Plaq.", obs[0].plaq);
        std::printf("\t%s\t = %g \n", "Topc.", obs[0].topc);
        std::printf("\t%s\t = %g \n", "Energ.", obs[0].energy);
        for (int i = 1; i < n_out && i < rows; i++) {  // OutputTerm::writeFlowObs (:75-84)
            std::printf("Flow Time %2.2lf\n", obs[i].t);
            std::printf("\t%s\t = %g \n", "Plaq.", obs[i].plaq);
            std::printf("\t%s\t = %g \n", "Topc.", obs[i].topc);
            std::printf("\t%s\t = %g \n", "Energ.", obs[i].energy);
        }
        char name[1024];
        std::snprintf(name, sizeof(name), "%s/flow/conf%04d.dat", in.output_dir.c_str(), conf_num);
        FILE* o = std::fopen(name, "w+");
        if (!o) die(std::string("cannot write ") + name);
        std::fprintf(o, "Flow Time\t");
        std::fprintf(o, "%s\t", "Plaq.");
        std::fprintf(o, "%s\t", "Topc.");
        std::fprintf(o, "%s\t", "Energ.");
        std::fprintf(o, "\n");
        for (int i = 0; i < rows && i < n_out; i++) {
            const double cells[4] = {obs[i].t, obs[i].plaq, obs[i].topc, obs[i].energy};
            for (double c : cells) std::fprintf(o, "%lf\t", c);
            std::fprintf(o, "\n");
        }
        std::fclose(o);
        std::snprintf(name, sizeof(name), "%s/flow/conf%04d.full.dat", in.output_dir.c_str(), conf_num);
        if (FILE* p = std::fopen(name, "w+")) {
            std::fprintf(p, "step\tt\tplaq\ttopc\tenergy\tt2E\n");
            for (int i = 0; i < rows && i < n_out; i++)
                std::fprintf(p, "%d\t%.17g\t%.17g\t%.17g\t%.17g\t%.17g\n", obs[i].step, obs[i].t, obs[i].plaq,
                             obs[i].topc, obs[i].energy, obs[i].t2E);
            std::fclose(p);
        }
        conf_num++;
    }
    for (ymflow_ctx* c : slabs) ymflow_destroy(c);
    const std::chrono::duration<double> el = std::chrono::system_clock::now() - start;
    std::printf("Total time taken: %.2fs\n", el.count());
    return 0;
}
