// ymflow_flow — drop-in replacement for the reference's LatticeQCD binary run
// with a FLOW or PGFG input file (src/MainPrograms/LatticeQCDMain.cpp:5-30), on B200s.
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
// (ymflow_slab_group_flow).  Any other split whose extents divide the lattice's
// flows as blocks in the reference's Cartesian layout, one per GPU
// round-robin (ymflow_create_block, ymflow_block_group_flow); each
// configuration file is read once and split among the blocks on the host.
//
// PGFG (the reference's gauge-field generator, src/Apps/gaugefieldfactory.cpp,
// whose update does not compile): the same App keys and validation
// (jsonapp.cpp:66-88, 103-118),
//   "App": {"type": "PGFG", "params": {"startType": "Cold"|"Hot", "MCSteps": M,
//           "thermSteps": T, "SU3eps": e, "NConf": n  or  "NCorr": c}}
// with NConf = MCSteps / NCorr when NCorr is given and MCSteps / NConf sweeps
// between configurations (gaugefieldfactory.cpp constructor), the same loops:
// thermSteps sweeps with a report every MCSteps / NConf, then MCSteps sweeps
// saving OutputDir/confNNNN.bin (outputconf.cpp:89-91, the .bin layout the FLOW
// app reads) and appending to OutputDir/observables.dat at each multiple of
// MCSteps / NConf (gaugefieldfactory.cpp:97-130).  The sweeps run on the device
// (ymflow_generate_metropolis: checkerboard Metropolis of the action's beta,
// 30 hits per link as gaugefieldfactory.cpp:210, seeded).  The reference prints
// and writes Observable::value(), which SuperObs leaves 0 (superobs.cpp:32);
// these lines and rows carry SuperObs' plaquette, charge and energy instead,
// and OutputDir/observables.full.dat repeats them at full precision with the
// acceptance.  "Hot" is Haar-random SU(3).  Optional keys: "Seed" (default 1),
// "MetropolisHits" (default 30).  InputDir is not read (jsondirectories.cpp:20-31).
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
    bool generate = false;  // App "PGFG" (else "FLOW")
    double epsilon = 0.0, tau_final = 0.0, beta = 0.0;
    // PGFG
    int mc_steps = 0, therm_steps = 0, corr_steps = 0, hits = 30;
    double su3eps = 0.0;
    bool hot = false, measure = false;
    uint64_t seed = 1;
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
    const jl::Value& params = app["params"];
    if (app["type"].is_string("PGFG")) {
        in.generate = true;
        if (params.size() != 5 || params["startType"].size() != 1 || params["MCSteps"].size() != 1 ||
            params["thermSteps"].size() != 1 || params["SU3eps"].size() != 1 ||
            params["NConf"].size() + params["NCorr"].size() != 1)
            die("wrong \"PGFG\" app specification\nCorrect format:\"App\" : {\n   \"type\" : \"PGFG\", \n"
                "   \"params\" : { \n       \"MCSteps\"   :  MCSteps, \n       \"themSteps\" :  thermSteps\n"
                "       \"startType\" :  startType, \n       \"NConf\"     : NConf,   OR    \"NCorr\" : NCorr, \n"
                "       \"SU3eps\"    : SU3eps \n   }\n}");
        const std::string start = params["startType"].kind == jl::Value::String ? params["startType"].str : "";
        if (start != "Cold" && start != "Hot") die("startType must be \"Cold\" or \"Hot\"");
        in.hot = start == "Hot";
        in.mc_steps = int(params["MCSteps"].num);
        in.therm_steps = int(params["thermSteps"].num);
        in.su3eps = params["SU3eps"].num;
        // registerPGFG (jsonapp.cpp:103-118) and the GaugeFieldFactory constructor
        int nconf = 0;
        if (params["NConf"].size() == 1) {
            nconf = int(params["NConf"].num);
        } else {
            const int ncorr = int(params["NCorr"].num);
            if (ncorr < 1) die("NCorr must be >= 1");
            nconf = in.mc_steps / ncorr;
        }
        if (in.mc_steps < 1 || in.therm_steps < 0) die("need MCSteps >= 1 and thermSteps >= 0");
        if (nconf < 1 || in.mc_steps / nconf < 1) die("need 1 <= NConf <= MCSteps");
        in.corr_steps = in.mc_steps / nconf;
        if (!(in.su3eps > 0.0 && in.su3eps < 1.0)) die("SU3eps must lie in (0, 1)");
    } else if (app["type"].is_string("FLOW")) {
        if (params.size() != 2 || params["epsilon"].size() != 1 || params["tauFinal"].size() != 1)
            die("wrong \"FLOW\" app specification\nCorrect format:\"App\" : {\n   \"type\" : \"FLOW\", \n"
                "   \"params\" : { \n       \"epsilon\" : epsilon, \n       \"tauFinal\" : tauFinal \n   }\n}");
        in.epsilon = params["epsilon"].num;
        in.tau_final = params["tauFinal"].num;
        if (!(in.epsilon > 0.0) || !(in.tau_final >= 0.0)) die("epsilon must be > 0 and tauFinal >= 0");
    } else if (app["type"].is_string("GFR")) {
        die("App \"GFR\" is not part of this drop-in (the reference's GaugeFieldReader::navigateConf is empty); "
            "\"FLOW\" and \"PGFG\" are provided");
    } else {
        die("unknown App " + (app["type"].kind == jl::Value::String ? app["type"].str : std::string("?")));
    }
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
    if (!superobs && !in.generate) die("FLOW measures through \"superobs\"; add it to Observables");
    in.measure = superobs;  // the reference registers only "superobs" (jsonobservable.cpp:64-78)
    // directories (jsondirectories.cpp:20-55); the generator reads no InputDir
    if (!in.generate && root.count("InputDir") == 0) die("no InputDir specified");
    if (root.count("OutputDir") == 0) die("no OutputDir specified");
    if (!in.generate) in.input_dir = root["InputDir"].str;
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
    if (root.count("Seed")) {
        if (root["Seed"].kind != jl::Value::Number || root["Seed"].num < 0) die("Seed must be a number >= 0");
        in.seed = uint64_t(root["Seed"].num);
    }
    if (root.count("MetropolisHits")) {
        in.hits = int(root["MetropolisHits"].num);
        if (in.hits < 1) die("MetropolisHits must be >= 1");
    }
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

// OutputDir/confNNNN.bin (OutputConf::writeConf, outputconf.cpp:80-104, whose
// write is commented out): the links in the .bin layout the FLOW app reads,
// streamed from the device in chunks of IOChunkSites sites.
void write_conf(ymflow_ctx* ctx, const Input& in, int conf_num) {
    char name[1024];
    std::snprintf(name, sizeof(name), "%s/conf%04d.bin", in.output_dir.c_str(), conf_num);
    FILE* f = std::fopen(name, "wb");
    if (!f) die(std::string("cannot write ") + name);
    const int64_t vol = int64_t(in.size[0]) * in.size[1] * in.size[2] * in.size[3];
    const int64_t chunk = std::min<int64_t>(in.chunk_sites, vol);
    std::vector<double> buf(static_cast<size_t>(chunk) * 72);
    for (int64_t s = 0; s < vol; s += chunk) {
        const int64_t n = std::min(chunk, vol - s);
        check(ymflow_download_sites(ctx, buf.data(), s, n, in.big_endian ? YMFLOW_IO_BIG_ENDIAN : 0), ctx,
              "download");
        if (std::fwrite(buf.data(), sizeof(double) * 72, size_t(n), f) != size_t(n))
            die(std::string("short write to ") + name);
    }
    if (std::fclose(f) != 0) die(std::string("cannot close ") + name);
}

// The PGFG application: GaugeFieldFactory::execute (gaugefieldfactory.cpp:62-108,
// 114-130) with its sweeps on the device.
void run_generator(const Input& in) {
    std::printf("Number of Processors: \t\t%i\n", 1);  // the lattice is generated whole on one GPU
    std::printf("Number of Active Processors: \t%i\n\n", 1);
    mkdir(in.output_dir.c_str(), 0755);  // OutputObs::setOutputDir creates both (outputobs.cpp:19-22)
    mkdir((in.output_dir + "/flow").c_str(), 0755);
    const std::string obs_path = in.output_dir + "/observables.dat";
    FILE* o = std::fopen(obs_path.c_str(), "w+");  // OutputObs::initialize (outputobs.cpp:29-39)
    if (!o) die("cannot write " + obs_path);
    std::fprintf(o, "Step\t");
    if (in.measure) std::fprintf(o, "%s\t%s\t%s\t", "Plaq.", "Topc.", "Energ.");
    std::fprintf(o, "\n");
    std::fclose(o);
    const std::string full_path = in.output_dir + "/observables.full.dat";
    FILE* p = std::fopen(full_path.c_str(), "w+");
    if (!p) die("cannot write " + full_path);
    std::fprintf(p, "step\tconf\tplaq\ttopc\tenergy\tacceptance\n");

    int st = 0;
    ymflow_ctx* ctx = ymflow_create(in.size, in.precision, in.device, &st);
    if (!ctx) die(std::string("ymflow_create: ") + ymflow_last_error(nullptr));
    const double tries_per_sweep = double(in.hits) * 4.0 * double(in.size[0]) * in.size[1] * in.size[2] * in.size[3];
    double accepted = 0.0, tries = 0.0;  // cumulative, as m_accepted / m_updates
    auto sweeps = [&](int start, int n) {
        double frac = 0.0;
        check(ymflow_generate_metropolis(ctx, start, in.beta, in.su3eps, n, in.hits, in.seed, &frac), ctx,
              "metropolis");
        accepted += std::round(frac * n * tries_per_sweep);
        tries += n * tries_per_sweep;
    };
    // OutputTerm::printThermStep / printGenStep (outputterm.cpp:29-51)
    auto report = [&](const char* head, int num) {
        ymflow_obs ob{};
        std::printf(head, num);
        if (in.measure) {
            check(ymflow_observables(ctx, &ob), ctx, "observables");
            std::printf("\t%s\t = %lf \n", "Plaq.", ob.plaq);
            std::printf("\t%s\t = %lf \n", "Topc.", ob.topc);
            std::printf("\t%s\t = %lf \n", "Energ.", ob.energy);
        }
        std::printf("\tAccept. Ratio = %lf\n", accepted / tries);
        return ob;
    };

    sweeps(in.hot ? YMFLOW_FIELD_HOT : YMFLOW_FIELD_COLD, 0);  // initialize (gaugefieldfactory.cpp:62-73)
    const int k = in.corr_steps;
    for (int step = k; step <= in.therm_steps; step += k) {  // thermalize (:97-108)
        sweeps(YMFLOW_FIELD_CURRENT, k);
        report("Thermalization Step %4i\n", step);
    }
    if (in.therm_steps % k) sweeps(YMFLOW_FIELD_CURRENT, in.therm_steps % k);
    // sampleConf (:114-130).  Sweeps after the last saved configuration change
    // no output and are not run.
    int conf_num = 0;
    for (int step = k; step <= in.mc_steps; step += k) {
        sweeps(YMFLOW_FIELD_CURRENT, k);
        const ymflow_obs ob = report("Configuration Number %4i\n", conf_num);
        if (FILE* w = std::fopen(obs_path.c_str(), "a")) {  // OutputObs::writeObs (outputobs.cpp:47-57)
            std::fprintf(w, "%i\t", step);
            if (in.measure) std::fprintf(w, "%lf\t%lf\t%lf\t", ob.plaq, ob.topc, ob.energy);
            std::fprintf(w, "\n");
            std::fclose(w);
        }
        std::fprintf(p, "%d\t%d\t%.17g\t%.17g\t%.17g\t%.17g\n", step, conf_num, ob.plaq, ob.topc, ob.energy,
                     accepted / tries);
        std::fflush(p);
        write_conf(ctx, in, conf_num);
        conf_num++;
    }
    std::fclose(p);
    ymflow_destroy(ctx);
}

}  // namespace

int main(int argc, char** argv) {
    const auto start = std::chrono::system_clock::now();
    if (argc != 2) die("wrong numper of command line arguments provided.");
    const Input in = parse_input(argv[1]);

    std::printf("Total Lattice Size: %2i %2i %2i %2i\n", in.size[0], in.size[1], in.size[2], in.size[3]);
    std::printf("Sublattice Size:    %2i %2i %2i %2i\n\n", in.sub[0], in.sub[1], in.sub[2], in.sub[3]);
    if (in.generate) {
        run_generator(in);
        const std::chrono::duration<double> el = std::chrono::system_clock::now() - start;
        std::printf("Total time taken: %.2fs\n", el.count());
        return 0;
    }
    // time slabs when SubLatticeSize splits only t, blocks for any other divisible split
    int nslabs = 1, nblocks = 0;
    int grid[4] = {1, 1, 1, 1};
    bool divides = true, spatial_split = false;
    for (int d = 0; d < 4; d++) {
        divides = divides && in.sub[d] >= 1 && in.size[d] % in.sub[d] == 0;
        if (d < 3 && in.sub[d] < in.size[d]) spatial_split = true;
    }
    if (divides && !spatial_split && in.sub[3] < in.size[3]) {
        if ((int64_t(in.size[0]) * in.size[1] * in.size[2]) % 32 == 0) {
            nslabs = in.size[3] / in.sub[3];
        } else {
            for (int d = 0; d < 4; d++) grid[d] = in.size[d] / in.sub[d];
            nblocks = grid[3];
        }
    } else if (divides && spatial_split) {
        nblocks = 1;
        for (int d = 0; d < 4; d++) {
            grid[d] = in.size[d] / in.sub[d];
            nblocks *= grid[d];
        }
    }
    const int nranks = nblocks > 0 ? nblocks : nslabs;
    std::printf("Number of Processors: \t\t%i\n", nranks);
    std::printf("Number of Active Processors: \t%i\n\n", nranks);

    mkdir(in.output_dir.c_str(), 0755);
    mkdir((in.output_dir + "/flow").c_str(), 0755);
    if (FILE* o = std::fopen((in.output_dir + "/observables.dat").c_str(), "w+")) {
        std::fprintf(o, "Step\t");
        std::fprintf(o, "%s\t", "SuperObs");
        std::fprintf(o, "\n");
        std::fclose(o);
    }

    int st = 0;
    std::vector<ymflow_ctx*> slabs;  // one context per slab or block (one: the whole lattice)
    if (nblocks > 0) {
        int ndev = 0;
        ymflow_device_count(&ndev);
        for (int i = 0; i < nblocks; i++) {  // block i at grid coordinates (i % g0, i / g0 % g1, ...)
            int origin[4], k = i;
            for (int d = 0; d < 4; d++) {
                origin[d] = (k % grid[d]) * in.sub[d];
                k /= grid[d];
            }
            const int dev = ndev > 0 ? (in.device + i) % ndev : in.device;
            ymflow_ctx* c = ymflow_create_block(in.size, origin, in.sub, in.precision, dev, &st);
            if (!c) die(std::string("ymflow_create_block: ") + ymflow_last_error(nullptr));
            slabs.push_back(c);
        }
    } else if (nslabs == 1) {
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
    std::vector<double> whole, part;
    for (const std::string& path : input_list(in.input_dir)) {
        if (nblocks > 0) {  // the file once, each block's own sites out of it (bytes as stored)
            const int64_t V = int64_t(in.size[0]) * in.size[1] * in.size[2] * in.size[3];
            whole.resize(size_t(V) * 72);
            FILE* fin = std::fopen(path.c_str(), "rb");
            if (!fin || std::fread(whole.data(), sizeof(double), whole.size(), fin) != whole.size() ||
                std::fgetc(fin) != EOF)
                die("configuration file " + path + " does not hold the lattice's links");
            std::fclose(fin);
            const int64_t bv = int64_t(in.sub[0]) * in.sub[1] * in.sub[2] * in.sub[3];
            part.resize(size_t(bv) * 72);
            for (int i = 0; i < nblocks; i++) {
                int origin[4], k = i;
                for (int d = 0; d < 4; d++) {
                    origin[d] = (k % grid[d]) * in.sub[d];
                    k /= grid[d];
                }
                size_t o = 0;
                for (int t = 0; t < in.sub[3]; t++)
                    for (int z = 0; z < in.sub[2]; z++)
                        for (int y = 0; y < in.sub[1]; y++) {  // one run of x per (t, z, y)
                            const int64_t s0 =
                                origin[0] + int64_t(in.size[0]) *
                                                (origin[1] + y + int64_t(in.size[1]) *
                                                                     (origin[2] + z + int64_t(in.size[2]) * (origin[3] + t)));
                            std::memcpy(part.data() + o, whole.data() + s0 * 72, size_t(in.sub[0]) * 72 * sizeof(double));
                            o += size_t(in.sub[0]) * 72;
                        }
                check(ymflow_upload_sites(slabs[i], part.data(), 0, bv, in.big_endian ? YMFLOW_IO_BIG_ENDIAN : 0),
                      slabs[i], "upload");
            }
        } else {
            for (ymflow_ctx* c : slabs)  // each slab reads its own part of the file
                check(ymflow_load_file(c, path.c_str(), in.big_endian ? YMFLOW_IO_BIG_ENDIAN : 0, in.chunk_sites), c,
                      "load");
        }
        int n_out = 0;
        if (nblocks > 0)
            check(ymflow_block_group_flow(slabs.data(), nblocks, grid, in.epsilon, nsteps, 1, in.reunit_every,
                                          obs.data(), int(obs.size()), &n_out),
                  ctx, "flow");
        else if (nslabs == 1)
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
