// gft_run.cpp -- GFTEvolver's main(), with the time loop on the GPU.
//
// Reads a configuration tree laid out like the reference's
// (<root>/Core/Config/Lattice.cfg, Model.cfg, Potentials/Config/*.cfg,
// WilsonLoops/Config/*.cfg, Analysers/Config/*.cfg), evolves through the C ABI
// of libgft_b200.so and writes what the reference's analysers write into
// <root>/Data: the Energy and GaugeCondition global-quantity rows
// (Analysers/Source/Energy.cpp:169-188, Analysers/Source/GaugeCondition.cpp:167-193)
// and the OutputFields dumps (Analysers/Source/OutputFields.cpp:63-133).  The
// reference's main() (main.cpp:10-60) constructs a Lattice, runs
// initialAnalysis, evolve, finalAnalysis; this program does the same three
// phases with Lattice::evolve (Core/Source/Lattice.cpp:755-876) replaced by
// gft_evolve.
//
// The .cfg files are positional, as the reference's configure() functions read
// them: a fixed number of description lines, then one entry per line whose
// values follow the last ':' of the line.
//
// Initial data: by default the configured one, built as the reference builds it
// (Lattice.cfg initial-condition types: 0 = zero scalars and identity links,
// 1 = RandomUniform from InitialConditions/Config/RandomUniform.cfg, a
// std::mt19937 stream per array); or --ic FILE (both time levels in the
// reference layout, float for the ref32 / mixed forms, double for ref64 / fp64);
// or --device-ic SEED (gft_init_fields: Higgs N(1, 0.1^2) per component, random
// links with eps, theta_Y ~ N(0, 0.1^2)).
//
// Usage: gft_run ROOT [--form ref32|ref64|fp64|mixed] [--ic FILE | --device-ic SEED]
//                     [--device N] [--initial-bin FILE [--initial-only]] [--final-bin FILE]
//                     [--print-config]
// --initial-only writes the host-built initial data to --initial-bin and exits
// without opening a device.
#include <cmath>
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <random>
#include <iostream>
#include <mutex>
#include <sstream>
#include <stdexcept>
#include <string>
#include <sys/stat.h>
#include <thread>
#include <vector>

#include "gft.h"

namespace {

using Entries = std::vector<std::vector<std::string>>;

// Entries of a positional .cfg file: after `header` description lines, the
// whitespace-separated tokens after the last ':' of every line that has one.
Entries read_cfg(const std::string& path, int header)
{
    std::ifstream f(path);
    if (!f) throw std::runtime_error("cannot open " + path);
    Entries out;
    std::string line;
    for (int i = 0; i < header && std::getline(f, line); i++) {
    }
    while (std::getline(f, line)) {
        const auto c = line.rfind(':');
        if (c == std::string::npos) continue;
        std::istringstream is(line.substr(c + 1));
        std::vector<std::string> tok;
        std::string t;
        while (is >> t) tok.push_back(t);
        out.push_back(tok);
    }
    return out;
}

const std::string& tok(const Entries& e, size_t i, size_t k, const std::string& file)
{
    if (i >= e.size() || k >= e[i].size())
        throw std::runtime_error(file + ": entry " + std::to_string(i) + " value " + std::to_string(k) + " missing");
    return e[i][k];
}
double num(const Entries& e, size_t i, size_t k, const std::string& file) { return std::stod(tok(e, i, k, file)); }
int inum(const Entries& e, size_t i, size_t k, const std::string& file) { return std::stoi(tok(e, i, k, file)); }

struct Analysers {
    bool energy = false, gauss = false, fields = false;
    std::string energy_path, gauss_path;
    bool energy_opt[6] = {};
    bool gauss_opt[2] = {};
    int energy_freq = 1, gauss_freq = 1;
    // local (per-site) outputs: Energy's six densities, GaugeCondition's violations
    bool energy_local_opt[6] = {};
    bool gauss_local = false;
    std::string energy_local_path, gauss_local_path;
    bool fields_both = false, fields_initial = false, fields_final = false, fields_continual = false;
    int fields_freq = 1;
    std::string fields_initial_path, fields_continual_path, fields_final_path;
};

// The reference's configured initial condition (Core/Source/Lattice.cpp:172-215, 358-401):
// type 0 = zero scalars / identity links, type 1 = RandomUniform
// (InitialConditions/Source/RandomUniform.cpp:60-77).
struct RefIC {
    int type[2] = {0, 0};
    unsigned seed = 0;
    float lo = 0.f, hi = 0.f;  // parsed as float, as RandomUniform.cpp:28 reads them
    bool equal = false;
};

struct Run {
    gft_config cfg{};
    int nt = 0;
    Analysers an;
    RefIC ic;
};

Run configure(const std::string& root)
{
    Run r;
    gft_config& c = r.cfg;
    // Core/Config/Lattice.cfg (Core/Source/Lattice.cpp:47-143)
    const std::string lat = root + "/Core/Config/Lattice.cfg";
    const Entries L = read_cfg(lat, 10);
    c.nx = inum(L, 0, 0, lat);
    c.ny = inum(L, 0, 1, lat);
    c.nz = inum(L, 0, 2, lat);
    c.dx = num(L, 1, 0, lat);
    c.dy = num(L, 1, 1, lat);
    c.dz = num(L, 1, 2, lat);
    r.nt = inum(L, 2, 0, lat);
    c.dt = num(L, 3, 0, lat);
    const int nsc = inum(L, 4, 0, lat);
    const int nvec = inum(L, 5, 0, lat);
    if (inum(L, 6, 0, lat)) {  // nt from light-crossing times (Lattice.cpp:78-87)
        const float crossings = (float)num(L, 7, 0, lat);
        r.nt = static_cast<int>(crossings * static_cast<float>(c.nx) * c.dx / (2 * c.dt));
    }
    r.ic.type[0] = inum(L, 8, 0, lat);
    r.ic.type[1] = inum(L, 8, 1, lat);
    if (r.ic.type[0] == 1 || r.ic.type[1] == 1) {
        const std::string rf = root + "/InitialConditions/Config/RandomUniform.cfg";
        const Entries R = read_cfg(rf, 12);
        r.ic.seed = (unsigned)std::stoul(tok(R, 0, 0, rf));
        r.ic.lo = std::stof(tok(R, 1, 0, rf));
        r.ic.hi = std::stof(tok(R, 1, 1, rf));
        r.ic.equal = inum(R, 2, 0, rf) != 0;
    }
    r.an.fields = inum(L, 9, 0, lat) != 0;
    r.an.energy = inum(L, 10, 0, lat) != 0;
    r.an.gauss = inum(L, 11, 0, lat) != 0;
    // faces (-x) (+x) (-y) (+y) (-z) (+z): per axis both periodic (3) or both Fixed (1)
    // (Core/Source/Lattice.cpp:217-258 requires periodic faces in pairs)
    for (int a = 0; a < 3; a++) {
        const int lo = inum(L, 12, 2 * a, lat), hi = inum(L, 12, 2 * a + 1, lat);
        if (lo == 1 && hi == 1)
            c.fixed_axes |= 1 << a;
        else if (lo != 3 || hi != 3)
            throw std::runtime_error("faces of axis " + std::to_string(a) +
                                     ": only periodic (3 3) or Fixed (1 1) pairs run on the GPU");
    }

    // Core/Config/Model.cfg (Core/Source/Model.cpp:173-221)
    const std::string mod = root + "/Core/Config/Model.cfg";
    const Entries M = read_cfg(mod, 11);
    const int pot = inum(M, 0, 0, mod), grad = inum(M, 1, 0, mod), wl = inum(M, 2, 0, mod);
    if (pot == 1 && grad == 2 && wl == 1 && nsc == 4)
        c.model = GFT_MODEL_SM;
    else if (pot == 2 && grad == 3 && wl == 2 && nsc == 8)
        c.model = GFT_MODEL_2HDM;
    else
        throw std::runtime_error("model (potential " + std::to_string(pot) + ", gradient " + std::to_string(grad) +
                                 ", wilson loop " + std::to_string(wl) + ", " + std::to_string(nsc) +
                                 " scalars) is not built for the GPU");

    c.damping = (float)num(M, 3, 0, mod);
    c.nt_damped = inum(M, 4, 0, mod);
    if (inum(M, 5, 0, mod)) c.nt_damped = static_cast<int>((float)num(M, 6, 0, mod) / c.dt);

    if (c.model == GFT_MODEL_SM) {
        // Potentials/Config/SO_N.cfg (Potentials/Source/SO_N.cpp:21-27)
        const std::string so = root + "/Potentials/Config/SO_N.cfg";
        const Entries S = read_cfg(so, 15);
        c.lambda = num(S, 0, 0, so);
        c.eta_sqr = num(S, 1, 0, so);
        // WilsonLoops/Config/StandardModel.cfg
        const std::string w = root + "/WilsonLoops/Config/StandardModel.cfg";
        const Entries W = read_cfg(w, 12);
        c.g = num(W, 0, 0, w);
        c.gp = num(W, 1, 0, w);
        c.div_tol = num(W, 2, 0, w);
    } else {
        // Potentials/Config/Double_SO_N.cfg (Potentials/Source/Double_SO_N.cpp:44-120)
        const std::string ds = root + "/Potentials/Config/Double_SO_N.cfg";
        const Entries D = read_cfg(ds, 40);
        if (inum(D, 0, 0, ds) != 4) throw std::runtime_error("Double_SO_N: only 4 + 4 components run on the GPU");
        c.apply_norm = inum(D, 1, 0, ds);
        c.energy_offset = num(D, 2, 0, ds);
        c.m1 = num(D, 3, 0, ds);
        c.m2 = num(D, 3, 1, ds);
        c.l1 = num(D, 4, 0, ds);
        c.l2 = num(D, 4, 1, ds);
        c.l3 = num(D, 5, 0, ds);
        c.break_son = inum(D, 6, 0, ds);
        c.m12r = num(D, 7, 0, ds);
        c.l4p5 = num(D, 8, 0, ds);
        c.l6r = num(D, 9, 0, ds);
        c.l7r = num(D, 9, 1, ds);
        c.break_uhalfn = inum(D, 10, 0, ds);
        c.m12i = num(D, 11, 0, ds);
        c.l4m5 = num(D, 12, 0, ds);
        c.l5i = num(D, 12, 1, ds);
        c.l6i = num(D, 13, 0, ds);
        c.l7i = num(D, 13, 1, ds);
        // WilsonLoops/Config/TwoHDM.cfg
        const std::string w = root + "/WilsonLoops/Config/TwoHDM.cfg";
        const Entries W = read_cfg(w, 12);
        c.g = num(W, 0, 0, w);
        c.gp = num(W, 1, 0, w);
        c.gpp = num(W, 2, 0, w);
        c.generator_rep = inum(W, 3, 0, w) != 0;
        c.div_tol = num(W, 4, 0, w);
    }
    // link words per direction (WilsonLoops/Source/StandardModel.cpp:195-210, TwoHDM.cpp:215-241):
    // SM 5 (quaternion) or 4 (generators); TwoHDM 5 / 6 / 9 (gaugeNum 4 / 5 / 7), or 4 / 5 / 7
    // with the generator representation
    if (c.model == GFT_MODEL_SM) {
        if (nvec == 4)
            c.generator_rep = 1;
        else if (nvec != 5)
            throw std::runtime_error("WilsonLoops::StandardModel needs 4 or 5 vector components per direction, not " +
                                     std::to_string(nvec));
    } else {
        const int lw = c.generator_rep ? 3 : 4;
        if (nvec == 1 + lw)
            c.higgs_family = GFT_HF_NONE;
        else if (nvec == 2 + lw)
            c.higgs_family = GFT_HF_U1;
        else if (nvec == 1 + 2 * lw)
            c.higgs_family = GFT_HF_SU2;
        else
            throw std::runtime_error("WilsonLoops::TwoHDM (" + std::string(c.generator_rep ? "generator" : "quaternion") +
                                     " representation) needs " + std::to_string(1 + lw) + ", " + std::to_string(2 + lw) +
                                     " or " + std::to_string(1 + 2 * lw) + " vector components per direction, not " +
                                     std::to_string(nvec));
    }

    // Analysers/Config/*.cfg (Analysers/Source/Energy.cpp:14-47, GaugeCondition.cpp:14-47, OutputFields.cpp:14-45)
    if (r.an.energy) {
        const std::string ef = root + "/Analysers/Config/Energy.cfg";
        const Entries E = read_cfg(ef, 13);
        r.an.energy_path = tok(E, 0, 0, ef);
        bool any = false;
        for (int k = 0; k < 6; k++) any |= (r.an.energy_opt[k] = inum(E, 1 + k, 0, ef) != 0);
        r.an.energy_freq = inum(E, 7, 0, ef);
        r.an.energy_local_path = tok(E, 8, 0, ef);
        bool any_local = false;
        for (int k = 0; k < 6; k++) any_local |= (r.an.energy_local_opt[k] = inum(E, 9 + k, 0, ef) != 0);
        c.energy_every = any ? r.an.energy_freq : 0;
        c.energy_local_every = any_local ? inum(E, 15, 0, ef) : 0;
    }
    if (r.an.gauss) {
        const std::string gf = root + "/Analysers/Config/GaugeCondition.cfg";
        const Entries G = read_cfg(gf, 13);
        r.an.gauss_path = tok(G, 0, 0, gf);
        r.an.gauss_opt[0] = inum(G, 1, 0, gf) != 0;
        r.an.gauss_opt[1] = inum(G, 2, 0, gf) != 0;
        r.an.gauss_freq = inum(G, 3, 0, gf);
        r.an.gauss_local_path = tok(G, 4, 0, gf);
        r.an.gauss_local = inum(G, 5, 0, gf) != 0;
        c.gauss_every = (r.an.gauss_opt[0] || r.an.gauss_opt[1]) ? r.an.gauss_freq : 0;
        c.gauss_local_every = r.an.gauss_local ? inum(G, 6, 0, gf) : 0;
    }
    if (r.an.fields) {
        const std::string of = root + "/Analysers/Config/OutputFields.cfg";
        const Entries O = read_cfg(of, 13);
        r.an.fields_both = inum(O, 0, 0, of) != 0;
        r.an.fields_initial = inum(O, 1, 0, of) != 0;
        r.an.fields_final = inum(O, 2, 0, of) != 0;
        r.an.fields_continual = inum(O, 3, 0, of) != 0;
        r.an.fields_freq = inum(O, 4, 0, of);
        r.an.fields_initial_path = tok(O, 5, 0, of);
        r.an.fields_continual_path = tok(O, 6, 0, of);
        r.an.fields_final_path = tok(O, 7, 0, of);
    }
    return r;
}

void check(int rc, gft_handle* h, const char* what)
{
    if (rc < 0) throw std::runtime_error(std::string(what) + ": " + gft_last_error(h));
    if (rc & GFT_W_ASIN_DOMAIN) std::cerr << "Panic: asin argument outside [-1, 1]\n";
    if (rc & GFT_W_SQRT_DOMAIN) std::cerr << "Panic: sqrt of a negative number\n";
    if (rc & GFT_W_NONFINITE) std::cerr << "Panic: non-finite field value\n";
}

// OutputFields::outputFields: one line per site, scalar then vector components.
template <class T>
void dump_fields(const std::string& path, const std::vector<T>& sc, const std::vector<T>& ve, int nsc, int time_step,
                 bool both)
{
    std::ofstream ofs(path);
    if (!ofs) throw std::runtime_error("cannot open for writing");
    const size_t nsite2 = sc.size() / nsc;
    const size_t nve = ve.size() / nsite2;
    const size_t n = both ? nsite2 : nsite2 / 2;
    const size_t t0 = both ? 0 : (size_t)((time_step + 1) % 2) * n;
    for (size_t s = t0; s < t0 + n; s++) {
        for (int k = 0; k < nsc; k++) ofs << sc[s * nsc + k] << " ";
        for (size_t k = 0; k < nve; k++) ofs << ve[s * nve + k] << " ";
        ofs << std::endl;
    }
}

// OutputFields dumps written by a background thread, so that formatting and
// writing the text of one dump overlaps the evolution to the next one.  One
// dump is in flight at most: submit() waits for the previous one, then swaps
// the caller's buffers with the writer's (the caller gets the previous, written
// buffers back, resized, to download into).
template <class T>
class FieldWriter {
public:
    FieldWriter() : worker_([this] { loop(); }) {}
    ~FieldWriter() { finish(); }

    void submit(const std::string& path, std::vector<T>& sc, std::vector<T>& ve, int nsc, int time_step, bool both)
    {
        std::unique_lock<std::mutex> lk(mu_);
        cv_.wait(lk, [&] { return !busy_; });
        if (!err_.empty()) throw std::runtime_error(err_);
        path_ = path;
        sc_.swap(sc);
        ve_.swap(ve);
        sc.resize(sc_.size());
        ve.resize(ve_.size());
        nsc_ = nsc;
        step_ = time_step;
        both_ = both;
        busy_ = true;
        cv_.notify_all();
    }

    // Waits for the last dump and stops the thread; returns the first write error ("" if none).
    std::string finish()
    {
        {
            std::unique_lock<std::mutex> lk(mu_);
            cv_.wait(lk, [&] { return !busy_; });
            stop_ = true;
        }
        cv_.notify_all();
        if (worker_.joinable()) worker_.join();
        return err_;
    }

private:
    void loop()
    {
        std::unique_lock<std::mutex> lk(mu_);
        for (;;) {
            cv_.wait(lk, [&] { return busy_ || stop_; });
            if (!busy_) return;
            lk.unlock();
            std::string e;
            try {
                dump_fields(path_, sc_, ve_, nsc_, step_, both_);
            } catch (const std::exception& ex) {
                e = ex.what();
            }
            lk.lock();
            if (!e.empty() && err_.empty()) err_ = "OutputFields " + path_ + ": " + e;
            busy_ = false;
            cv_.notify_all();
        }
    }

    std::mutex mu_;
    std::condition_variable cv_;
    bool busy_ = false, stop_ = false;
    std::string err_, path_;
    std::vector<T> sc_, ve_;
    int nsc_ = 0, step_ = 0;
    bool both_ = false;
    std::thread worker_;
};

// Link words per site and gauge equations per direction of a configuration.
int vector_words(const gft_config& c)
{
    const int lw = c.generator_rep ? 3 : 4;
    return 3 * (1 + lw + (c.higgs_family == GFT_HF_U1 ? 1 : (c.higgs_family == GFT_HF_SU2 ? lw : 0)));
}
int gauss_count(const gft_config& c) { return c.higgs_family == GFT_HF_U1 ? 5 : (c.higgs_family == GFT_HF_SU2 ? 7 : 4); }

// RandomUniform::setInitialFields: one std::mt19937 stream per field array from
// the configured seed, float uniform in [lo, hi) as the reference stores it
// (widened exactly for the FP64 forms), both time levels equal when asked.
template <class T>
void random_uniform(std::vector<T>& field, const RefIC& ic)
{
    std::mt19937 generator(ic.seed);
    std::uniform_real_distribution<float> distribution(ic.lo, ic.hi);
    size_t n = field.size();
    if (ic.equal) n /= 2;
    for (size_t i = 0; i < n; i++) {
        field[i] = (T)distribution(generator);
        if (ic.equal) field[i + n] = field[i];
    }
}

template <class T>
void write_bin(const std::string& path, const std::vector<T>& sc, const std::vector<T>& ve)
{
    std::ofstream f(path, std::ios::binary);
    f.write(reinterpret_cast<const char*>(sc.data()), sc.size() * sizeof(T));
    f.write(reinterpret_cast<const char*>(ve.data()), ve.size() * sizeof(T));
    if (!f) throw std::runtime_error("cannot write " + path);
}

// Host-side initial data: the --ic file, or the configured initial condition
// built as the reference builds it.  Both time levels, reference layout.
template <class T>
void host_initial(const Run& r, const std::string& ic_path, std::vector<T>& sc, std::vector<T>& ve)
{
    if (!ic_path.empty()) {
        std::ifstream f(ic_path, std::ios::binary);
        f.read(reinterpret_cast<char*>(sc.data()), sc.size() * sizeof(T));
        f.read(reinterpret_cast<char*>(ve.data()), ve.size() * sizeof(T));
        if (!f) throw std::runtime_error("short initial-data file " + ic_path);
        return;
    }
    std::fill(sc.begin(), sc.end(), (T)0);
    std::fill(ve.begin(), ve.end(), (T)0);
    // zero gauge field: identity quaternions (Core/Source/Lattice.cpp:369-395); all zero generators
    const int nve = vector_words(r.cfg), dw = nve / 3;
    if (!r.cfg.generator_rep)
        for (size_t s = 0; s < ve.size() / nve; s++)
            for (int d = 0; d < 3; d++) {
                ve[s * nve + d * dw + 1] = (T)1;               // identity isospin link
                if (dw == 9) ve[s * nve + d * dw + 5] = (T)1;  // identity Higgs-family SU(2) link
            }
    if (r.ic.type[0] == 1) random_uniform(sc, r.ic);
    if (r.ic.type[1] == 1) random_uniform(ve, r.ic);
}

template <class T>
int run(const std::string& root, Run& r, const std::string& ic_path, long long seed, const std::string& final_bin,
        const std::string& initial_bin, bool initial_only)
{
    gft_config& c = r.cfg;
    const int nsc = (c.model == GFT_MODEL_SM) ? 4 : 8;
    const size_t nsite = (size_t)c.nx * c.ny * c.nz;
    std::vector<T> sc(2 * nsite * nsc), ve(2 * nsite * vector_words(c));
    if (initial_only) {  // the host-built initial data alone, no device
        if (seed >= 0) throw std::runtime_error("--initial-only builds host initial data; drop --device-ic");
        host_initial(r, ic_path, sc, ve);
        write_bin(initial_bin, sc, ve);
        return 0;
    }
    const std::string data = root + "/Data";
    mkdir(data.c_str(), 0755);
    for (const std::string* sub : {&r.an.fields_continual_path, &r.an.energy_local_path, &r.an.gauss_local_path}) {
        const auto slash = sub->rfind('/');
        if (slash != std::string::npos) mkdir((data + "/" + sub->substr(0, slash)).c_str(), 0755);
    }

    gft_handle* h = nullptr;
    check(gft_create(&c, &h), nullptr, "gft_create");
    auto download = [&]() {
        if constexpr (sizeof(T) == 4)
            check(gft_download_f32(h, sc.data(), ve.data()), h, "gft_download");
        else
            check(gft_download_f64(h, sc.data(), ve.data()), h, "gft_download");
    };
    if (seed < 0) {
        host_initial(r, ic_path, sc, ve);
        if constexpr (sizeof(T) == 4)
            check(gft_upload_f32(h, sc.data(), ve.data(), 0), h, "gft_upload");
        else
            check(gft_upload_f64(h, sc.data(), ve.data(), 0), h, "gft_upload");
    } else {
        gft_ic ic{};
        ic.seed = (uint64_t)seed;
        for (int k = 0; k < 8; k++) {
            ic.mean[k] = 1.0;
            ic.sigma[k] = 0.1;
        }
        ic.theta_sigma = 0.1;
        ic.eps_sigma = 0.1;
        check(gft_init_fields(h, &ic), h, "gft_init_fields");
    }

    // initialAnalysis (OutputFields, Analysers/Source/OutputFields.cpp:63-133, 155-200: text dumps in a
    // background thread)
    FieldWriter<T> writer;
    if ((r.an.fields && r.an.fields_initial) || !initial_bin.empty()) download();
    if (!initial_bin.empty()) write_bin(initial_bin, sc, ve);
    if (r.an.fields && r.an.fields_initial)
        writer.submit(data + "/" + r.an.fields_initial_path, sc, ve, nsc, 0, r.an.fields_both);

    // evolve: chunks end where OutputFields writes a continual dump or an analyser keeps its local outputs
    const int ffreq = (r.an.fields && r.an.fields_continual && r.an.fields_freq > 0) ? r.an.fields_freq : 0;
    const int lef = c.energy_local_every, lgf = c.gauss_local_every, neq = gauss_count(c);
    auto next_stop = [&](int d) {  // steps done at the end of the chunk that starts with d done
        int stop = std::min(r.nt, d + 1000);
        if (ffreq > 0) stop = std::min(stop, (d / ffreq + 1) * ffreq);
        for (int f : {lef, lgf})
            if (f > 0) stop = std::min(stop, (d + f - 1) / f * f + 1);  // after the next local-output step
        return stop;
    };
    std::vector<gft_observables> rows;
    std::vector<float> loc_e(lef > 0 ? nsite * 6 : 0), loc_g(lgf > 0 ? nsite * (size_t)neq : 0);
    int done = 0;
    while (done < r.nt) {
        const int n = next_stop(done) - done;
        rows.resize((size_t)n + 1);
        int got = 0;
        check(gft_evolve(h, n, rows.data(), (int)rows.size(), &got), h, "gft_evolve");
        done += n;
        for (int i = 0; i < got; i++) {
            const gft_observables& o = rows[i];
            if (o.has_energy && !r.an.energy_path.empty()) {
                std::ofstream ofs(data + "/" + r.an.energy_path, std::ios::app);
                const double v[6] = {o.energy, o.potential, o.gradient, o.kinetic, o.magnetic, o.electric};
                for (int k = 0; k < 6; k++)
                    if (r.an.energy_opt[k]) ofs << v[k] << " ";
                ofs << "\n";
            }
            if (o.has_gauss && !r.an.gauss_path.empty()) {
                std::ofstream ofs(data + "/" + r.an.gauss_path, std::ios::app);
                if (r.an.gauss_opt[0])
                    for (int k = 0; k < neq; k++) ofs << o.gauss_int[k] << " ";
                if (r.an.gauss_opt[1])
                    for (int k = 0; k < neq; k++) ofs << o.gauss_max[k] << " ";
                ofs << "\n";
            }
        }
        // local outputs of step done - 1 (Energy.cpp:191-207: option-major, one value per line;
        // GaugeCondition.cpp:194-212: site-major, gaugeNum values per site)
        const int last = done - 1;
        const bool le = lef > 0 && last % lef == 0, lg = lgf > 0 && last % lgf == 0;
        if (le || lg) {
            int es = -1, gs = -1;
            check(gft_local_fields(h, le ? loc_e.data() : nullptr, lg ? loc_g.data() : nullptr, &es, &gs), h,
                  "gft_local_fields");
            if (le) {
                std::ofstream ofs(data + "/" + r.an.energy_local_path + "_" + std::to_string(last) + ".dat");
                for (int k = 0; k < 6; k++)
                    if (r.an.energy_local_opt[k])
                        for (size_t s = 0; s < nsite; s++) ofs << loc_e[s * 6 + k] << "\n";
            }
            if (lg) {
                std::ofstream ofs(data + "/" + r.an.gauss_local_path + "_" + std::to_string(last) + ".dat");
                for (size_t k = 0; k < loc_g.size(); k++) ofs << loc_g[k] << "\n";
            }
        }
        if (ffreq > 0 && done % ffreq == 0) {
            download();
            writer.submit(data + "/" + r.an.fields_continual_path + "_" + std::to_string(done) + ".dat", sc, ve, nsc,
                          done, r.an.fields_both);
        }
    }

    // finalAnalysis
    download();
    if (!final_bin.empty()) write_bin(final_bin, sc, ve);
    if (r.an.fields && r.an.fields_final)
        writer.submit(data + "/" + r.an.fields_final_path, sc, ve, nsc, r.nt, r.an.fields_both);
    const std::string werr = writer.finish();
    gft_destroy(h);
    if (!werr.empty()) throw std::runtime_error(werr);
    return 0;
}

}  // namespace

int main(int argc, char** argv)
{
    if (argc < 2) {
        std::cerr << "usage: gft_run ROOT [--form ref32|ref64|fp64|mixed] [--ic FILE | --device-ic SEED] "
                     "[--device N] [--initial-bin FILE [--initial-only]] [--final-bin FILE] [--print-config]\n";
        return 2;
    }
    try {
        const std::string root = argv[1];
        std::string form = "mixed", ic, final_bin, initial_bin;
        long long seed = -1;
        int device = 0;
        bool print = false, initial_only = false;
        for (int i = 2; i < argc; i++) {
            const std::string a = argv[i];
            auto next = [&]() -> std::string {
                if (i + 1 >= argc) throw std::runtime_error(a + " needs a value");
                return argv[++i];
            };
            if (a == "--form") form = next();
            else if (a == "--ic") ic = next();
            else if (a == "--device-ic") seed = std::stoll(next());
            else if (a == "--device") device = std::stoi(next());
            else if (a == "--final-bin") final_bin = next();
            else if (a == "--initial-bin") initial_bin = next();
            else if (a == "--initial-only") initial_only = true;
            else if (a == "--print-config") print = true;
            else throw std::runtime_error("unknown option " + a);
        }
        Run r = configure(root);
        r.cfg.device = device;
        bool f64 = false;
        if (form == "ref32") { r.cfg.form = GFT_FORM_REF; r.cfg.storage_bytes = 4; }
        else if (form == "ref64") { r.cfg.form = GFT_FORM_REF; r.cfg.storage_bytes = 8; f64 = true; }
        else if (form == "fp64") { r.cfg.form = GFT_FORM_FP64; f64 = true; }
        else if (form == "mixed") { r.cfg.form = GFT_FORM_MIXED; }
        else throw std::runtime_error("unknown form " + form);
        if (print) {
            const gft_config& c = r.cfg;
            std::printf("model %d form %d storage %d nx %d ny %d nz %d dx %.17g dy %.17g dz %.17g dt %.17g nt %d\n",
                        c.model, c.form, c.storage_bytes, c.nx, c.ny, c.nz, c.dx, c.dy, c.dz, c.dt, r.nt);
            std::printf("g %.17g gp %.17g div_tol %.17g damping %.17g nt_damped %d lambda %.17g eta_sqr %.17g\n", c.g,
                        c.gp, c.div_tol, c.damping, c.nt_damped, c.lambda, c.eta_sqr);
            std::printf("m1 %.17g m2 %.17g l1 %.17g l2 %.17g l3 %.17g m12r %.17g l4p5 %.17g l6r %.17g l7r %.17g\n", c.m1,
                        c.m2, c.l1, c.l2, c.l3, c.m12r, c.l4p5, c.l6r, c.l7r);
            std::printf("m12i %.17g l4m5 %.17g l5i %.17g l6i %.17g l7i %.17g break_son %d break_uhalfn %d "
                        "apply_norm %d energy_offset %.17g\n",
                        c.m12i, c.l4m5, c.l5i, c.l6i, c.l7i, c.break_son, c.break_uhalfn, c.apply_norm,
                        c.energy_offset);
            std::printf("energy_every %d gauss_every %d energy_path %s gauss_path %s fixed_axes %d\n", c.energy_every,
                        c.gauss_every, r.an.energy_path.c_str(), r.an.gauss_path.c_str(), c.fixed_axes);
            std::printf("higgs_family %d gpp %.17g generator_rep %d\n", c.higgs_family, c.gpp, c.generator_rep);
            std::printf("energy_local_every %d gauss_local_every %d\n", c.energy_local_every, c.gauss_local_every);
            std::printf("ic_scalar %d ic_gauge %d ic_seed %u ic_min %.9g ic_max %.9g ic_equal %d\n", r.ic.type[0],
                        r.ic.type[1], r.ic.seed, r.ic.lo, r.ic.hi, (int)r.ic.equal);
            return 0;
        }
        if (initial_only && initial_bin.empty()) throw std::runtime_error("--initial-only needs --initial-bin FILE");
        return f64 ? run<double>(root, r, ic, seed, final_bin, initial_bin, initial_only)
                   : run<float>(root, r, ic, seed, final_bin, initial_bin, initial_only);
    } catch (const std::exception& e) {
        std::cerr << "Error in " << e.what() << std::endl;
        return 1;
    }
}
