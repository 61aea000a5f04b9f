/*
 * ref_harness.cpp -- TEST INFRASTRUCTURE ONLY.  Replaces the reference's
 * main.cpp (main.cpp:10-67) so that the unmodified reference can be run on
 * generated initial data and its results read back at full precision.
 *
 * Usage:  GFT_REF_WORKDIR=<dir> ref32|ref64
 *   <dir>/<Module>/Config/*.cfg   configuration (written by oracle/refrun.py)
 *   <dir>/ic.bin                  optional: both time levels, scalars then vectors,
 *                                 raw storage words in the reference layout (without
 *                                 it the configured initial condition stands)
 * Output:
 *   <dir>/initial.bin             the initial fields the run started from
 *   <dir>/final.bin               both time levels after nt steps (same layout)
 *   <dir>/rows.txt                per logged step: the Energy analyser's running
 *                                 sums and the GaugeCondition sums and maxima (7
 *                                 each, zero beyond gaugeNum), read before the
 *                                 analysers write and reset them
 *   <dir>/timing.txt              wall seconds of Lattice::evolve
 *
 * The analysers' sums are private members of the reference classes; this file
 * (and only this file) is compiled with `private`/`protected` mapped to
 * `public` after the standard headers, which changes no layout.
 */
#include "ref_shim.h"

#define private public
#define protected public
#include "Lattice.hpp"
#undef private
#undef protected

namespace {

typedef float word_t;  // float in the shipped build; double in the FP64 variant (shim)

class CaptureAnalyser : public Analyser
{
public:
    Energy* energy = nullptr;
    GaugeCondition* gauge = nullptr;
    std::ofstream out;

    void configure(const std::string, const bool) override {}
    void initialAnalysis() override {}
    void preEvolveLocationAnalysis(const long long unsigned, const float* const[2],
                                   const std::vector<std::vector<const float*>>&, const float* const[2],
                                   const std::vector<std::vector<const float*>>&) override {}
    void postEvolveLocationAnalysis(const unsigned&, const long long unsigned, const float* const[2],
                                    const std::vector<std::vector<const float*>>&, const float* const[2],
                                    const std::vector<std::vector<const float*>>&) override {}
    void finalAnalysis() override {}

    // Runs before the Energy and GaugeCondition timestepAnalysis of the same step.
    void timestepAnalysis(const unsigned& time_step) override
    {
        bool e = energy && energy->globalOutput;
        bool g = gauge && gauge->globalOutput;
        if (!e && !g) return;
        out << time_step << " " << (e ? 1 : 0) << " " << (g ? 1 : 0);
        out << std::setprecision(17);
        for (unsigned k = 0; k < 6; k++) out << " " << (e ? (double)*energy->energyPointers[k] : 0.0);
        // up to gaugeNum = 7 constraint equations (WilsonLoops/Source/TwoHDM.cpp:276-279), zero-padded
        for (unsigned k = 0; k < 7; k++)
            out << " " << (g && k < gauge->integratedAbsViolation.size() ? (double)gauge->integratedAbsViolation[k] : 0.0);
        for (unsigned k = 0; k < 7; k++)
            out << " " << (g && k < gauge->maxAbsViolation.size() ? (double)gauge->maxAbsViolation[k] : 0.0);
        out << "\n";
    }
};

}  // namespace

int main()
{
    try {
        const std::string work = gft_ref_workdir();
        std::filesystem::create_directories(std::filesystem::path(DATA_DIR));
        std::filesystem::create_directories(std::filesystem::path(DATA_DIR) / "Continual");

        Lattice lattice;

        // Initial data from ic.bin, when given, replaces the configured initial
        // condition; without it the configured one (Lattice.cfg types) stands.
        {
            std::ifstream ic(work + "/ic.bin", std::ios::binary);
            if (ic) {
                ic.read(reinterpret_cast<char*>(lattice.scalarFields.data()),
                        (std::streamsize)(lattice.scalarFields.size() * sizeof(word_t)));
                ic.read(reinterpret_cast<char*>(lattice.vectorFields.data()),
                        (std::streamsize)(lattice.vectorFields.size() * sizeof(word_t)));
                if (!ic) throw std::runtime_error("ref_harness: ic.bin is shorter than the configured lattice");
            }
            std::ofstream fi(work + "/initial.bin", std::ios::binary);
            fi.write(reinterpret_cast<const char*>(lattice.scalarFields.data()),
                     (std::streamsize)(lattice.scalarFields.size() * sizeof(word_t)));
            fi.write(reinterpret_cast<const char*>(lattice.vectorFields.data()),
                     (std::streamsize)(lattice.vectorFields.size() * sizeof(word_t)));
        }

        CaptureAnalyser* cap = new CaptureAnalyser();
        for (Analyser* a : lattice.analysers) {
            if (auto* e = dynamic_cast<Energy*>(a)) cap->energy = e;
            if (auto* g = dynamic_cast<GaugeCondition*>(a)) cap->gauge = g;
        }
        cap->out.open(work + "/rows.txt");
        lattice.analysers.insert(lattice.analysers.begin(), cap);

        lattice.initialAnalysis();
        auto t0 = std::chrono::steady_clock::now();
        lattice.evolve();
        auto t1 = std::chrono::steady_clock::now();
        lattice.finalAnalysis();
        cap->out.close();

        {
            std::ofstream fo(work + "/final.bin", std::ios::binary);
            fo.write(reinterpret_cast<const char*>(lattice.scalarFields.data()),
                     (std::streamsize)(lattice.scalarFields.size() * sizeof(word_t)));
            fo.write(reinterpret_cast<const char*>(lattice.vectorFields.data()),
                     (std::streamsize)(lattice.vectorFields.size() * sizeof(word_t)));
        }
        {
            std::ofstream ft(work + "/timing.txt");
            ft << std::setprecision(9) << std::chrono::duration<double>(t1 - t0).count() << " "
               << sizeof(word_t) << "\n";
        }
        return EXIT_SUCCESS;
    } catch (const std::exception& ex) {
        std::cerr << "Error in " << ex.what() << std::endl;
        return EXIT_FAILURE;
    }
}
