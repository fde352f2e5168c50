// The reference application's WilsonFlow (include/Apps/wilsonflow.h) with its
// flow and its measurements on a B200 through libymflow's C ABI.
//
// Linked into the reference's own LatticeQCD program in place of
// src/Apps/wilsonflow.cpp, it is what the reference's JSON layer creates for
// "App": {"type": "FLOW"} (src/InputOutput/JsonInput/JsonGeneric/jsonapp.cpp:124-128).
// The reference's reader fills the host field (InputConf::readConf) and its
// writers print and store the rows (OutputTerm, OutputObs); the field goes to
// the GPU once per configuration, and the RK3 steps and every measurement run
// there.  The class layout is the reference header's; these member
// definitions replace the reference's.
//
// Environment: YMFLOW_PRECISION = fp64 (default) | fp32_18 | fp32_12,
// YMFLOW_DEVICE (default 0), YMFLOW_REUNIT_EVERY (mixed forms, default 10).
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "lqcd.h"
#include "ymflow.h"

namespace {

ymflow_ctx* g_ctx = nullptr;  // the reference runs one WilsonFlow per process

[[noreturn]] void die(const std::string& what, int status) {
    std::fprintf(stderr, "ymflow %s: %s (status %d)\n", what.c_str(), ymflow_last_error(g_ctx), status);
    std::exit(1);
}

void check(int status, const char* what) {
    if (status != YMFLOW_OK) die(what, status);
}

int env_int(const char* name, int fallback) {
    const char* v = std::getenv(name);
    return v ? std::atoi(v) : fallback;
}

int env_precision() {
    const char* v = std::getenv("YMFLOW_PRECISION");
    if (!v || !std::strcmp(v, "fp64")) return YMFLOW_FP64;
    if (!std::strcmp(v, "fp32_18")) return YMFLOW_FP32_18;
    if (!std::strcmp(v, "fp32_12")) return YMFLOW_FP32_12;
    std::fprintf(stderr, "unknown YMFLOW_PRECISION \"%s\" (fp64, fp32_18, fp32_12)\n", v);
    std::exit(1);
}

// every observable of the application reports the GPU's values
void set_observables(std::vector<Observable*>& obs, double plaq, double topc, double energy) {
    for (Observable* o : obs) {
        o->plaq = plaq;
        o->topc = topc;
        o->energy = energy;
    }
}

void release() {
    ymflow_destroy(g_ctx);
    g_ctx = nullptr;
}

}  // namespace

WilsonFlow::WilsonFlow(double tauFinal, double epsilon) {
    m_epsilon = epsilon;
    m_tauFinal = tauFinal;
}

void WilsonFlow::execute() {
    initialize();
    flowConfigurations();
}

// The application's start-up, through the reference's own I/O (the same calls
// as its WilsonFlow, wilsonflow.cpp:58-66, so the files and lines it writes
// are the same).
void WilsonFlow::initialize() {
    for (Observable* o : m_obs) o->initObservable(m_lat);
    m_act->initAction(m_lat);
    m_obsValues.resize(m_obs.size());
    LatticeIO::InputConf::getInputList(m_inputConfList);
    LatticeIO::OutputObs::initialize(m_obs);
    LatticeIO::OutputTerm::printInitialConditions();
}

// The host field the reference's reader fills, and the device context.
void WilsonFlow::createLattice(std::array<int, 4> latticeSize) {
    m_size = latticeSize;
    m_lat = new GluonField(m_size);
    int status = 0;
    g_ctx = ymflow_create(m_size.data(), env_precision(), env_int("YMFLOW_DEVICE", 0), &status);
    if (!g_ctx) die("create", status);
    std::atexit(release);
}

void WilsonFlow::computeObservables() {
    ymflow_obs o;
    check(ymflow_observables(g_ctx, &o), "observables");
    set_observables(m_obs, o.plaq, o.topc, o.energy);
}

void WilsonFlow::flowConfigurations() {
    if (!Parallel::isActive()) return;
    const int V = m_size[0] * m_size[1] * m_size[2] * m_size[3];
    std::vector<double> links(size_t(V) * 4 * 18);
    int confNum = 0;
    for (const std::string& conf : m_inputConfList) {
        LatticeIO::InputConf::readConf(*m_lat, conf.c_str());
        for (int s = 0; s < V; s++)  // .bin order: site, then direction, then 18 doubles
            for (int mu = 0; mu < 4; mu++)
                std::memcpy(&links[(size_t(s) * 4 + mu) * 18], (*m_lat)[mu].at(s).mat.data(), 18 * sizeof(double));
        check(ymflow_upload(g_ctx, links.data()), "upload");
        computeObservables();
        LatticeIO::OutputTerm::writeObs(confNum, m_obs);
        applyWilsonFlow(confNum);
        confNum++;
    }
}

// int(tauFinal/epsilon) rows, the first the configuration as read and one per
// flow step after it (wilsonflow.cpp:115-136); all steps run in one
// ymflow_flow call, measured after each.
void WilsonFlow::applyWilsonFlow(int confNum) {
    const int rows = int(m_tauFinal / m_epsilon) > 0 ? int(m_tauFinal / m_epsilon) : 1;
    std::vector<std::vector<double>> flowObs(rows, std::vector<double>(4, 0.0));
    flowObs[0] = {0.0, m_obs[0]->plaq, m_obs[0]->topc, m_obs[0]->energy};
    std::vector<ymflow_obs> out(rows + 1);
    int n = 0;
    const int reunit = env_int("YMFLOW_REUNIT_EVERY", 10);
    check(ymflow_flow(g_ctx, m_epsilon, rows - 1, 1, reunit, out.data(), rows + 1, &n), "flow");
    for (int t = 1; t < rows && t < n; t++) {
        flowObs[t] = {flowObs[t - 1][0] + m_epsilon, out[t].plaq, out[t].topc, out[t].energy};
        set_observables(m_obs, out[t].plaq, out[t].topc, out[t].energy);
        LatticeIO::OutputTerm::writeFlowObs(flowObs[t][0], m_obs);
    }
    LatticeIO::OutputObs::writeFlowObs(confNum, m_obs, flowObs);
}
