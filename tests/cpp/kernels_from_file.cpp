// Drives the C++ kernel classes of include/interax_b200_kernels.hpp the way a platform would: Force objects with the
// reference's accessors, a ContextAccess over plain arrays, the factory by kernel name.  Reads a system written by
// tests/test_cpp_kernels.py, writes the per-kernel energies and the summed forces.
//
//   kernels_from_file <input> <output>
#include <cstdio>
#include <fstream>
#include <iostream>
#include <memory>
#include <sstream>
#include <string>
#include <vector>

#include "interax_b200_kernels.hpp"

namespace {

// Force classes with the reference API's accessors (what the kernels need of them).
struct PairForce {
    int method = 0, group = 0, overlap = 0;
    double cutoff = 1.0, switchDist = -1.0, softcore = 0.0, damping = 1.0;
    bool useSwitch = false, lrc = false;
    std::string alchName = "lambda_sterics";
    int stride = 0;
    std::vector<double> params;
    std::vector<int> alch, excl;
    int getNumParticles() const { return (int)alch.size(); }
    int getNonbondedMethod() const { return method; }
    double getCutoffDistance() const { return cutoff; }
    bool getUseSwitchingFunction() const { return useSwitch; }
    double getSwitchingDistance() const { return switchDist; }
    double getSoftcoreRadius() const { return softcore; }
    int getForceGroup() const { return group; }
    const std::string& getAlchemicalParameterName() const { return alchName; }
    int getNumExclusions() const { return (int)excl.size() / 2; }
    void getExclusionParticles(int k, int& a, int& b) const {
        a = excl[2 * k];
        b = excl[2 * k + 1];
    }
    double getDampingScale() const { return damping; }
    bool getUseLongRangeCorrection() const { return lrc; }
    int getOverlapMethod() const { return overlap; }
    // dispersion, exchange, short range
    void getParticleParameters(int i, double& a, double& b, double& c, double& d, double& e, bool& al) const {
        a = params[5 * i], b = params[5 * i + 1], c = params[5 * i + 2], d = params[5 * i + 3], e = params[5 * i + 4];
        al = alch[i] != 0;
    }
    void getParticleParameters(int i, double& a, double& b, bool& al) const {
        a = params[2 * i], b = params[2 * i + 1];
        al = alch[i] != 0;
    }
    void getParticleParameters(int i, double& a, double& b, double& c, bool& al) const {
        a = params[3 * i], b = params[3 * i + 1], c = params[3 * i + 2];
        al = alch[i] != 0;
    }
};

struct ThreeBodyForce {
    double cutoff = 1.0, scale = 1.0, damping = 1.0, centroid = 0.0;
    int dampingMethod = 0, group = 0;
    bool periodic = false;
    std::string alchName = "lambda_sterics";
    std::vector<std::vector<int>> particles;
    std::vector<double> params;
    std::vector<int> molecule, alch;
    int getNumSites() const { return (int)molecule.size(); }
    void getSiteParameters(int s, std::vector<int>& p, double& alpha, double& freq, double& width, int& mol,
                           bool& al) const {
        p = particles[s];
        alpha = params[3 * s], freq = params[3 * s + 1], width = params[3 * s + 2];
        mol = molecule[s];
        al = alch[s] != 0;
    }
    double getCutoffDistance() const { return cutoff; }
    double getScaleFactor() const { return scale; }
    int getDampingMethod() const { return dampingMethod; }
    double getDampingScale() const { return damping; }
    double getCentroidDampingRadius() const { return centroid; }
    bool usesPeriodicBoundaryConditions() const { return periodic; }
    const std::string& getAlchemicalParameterName() const { return alchName; }
    int getForceGroup() const { return group; }
};

struct System {
    int n = 0;
    int getNumParticles() const { return n; }
};

// The platform side: arrays in place of OpenMM's ContextImpl.
struct ArrayContext : InteraxB200::ContextAccess {
    std::vector<double> pos, forces;
    double box[9] = {0};
    double lambda = 1.0;
    long long id = 0;
    int getNumParticles() const override { return (int)pos.size() / 3; }
    void getPositions(std::vector<double>& xyz) const override { xyz = pos; }
    void getPeriodicBoxVectors(double b[9]) const override {
        for (int k = 0; k < 9; k++) b[k] = box[k];
    }
    double getParameter(const std::string&) const override { return lambda; }
    long long getEvaluationId() const override { return id; }
    void addForces(const std::vector<double>& f) override {
        for (size_t k = 0; k < f.size(); k++) forces[k] += f[k];
    }
};

}  // namespace

template <class T>
void readVec(std::istream& in, std::vector<T>& v, size_t n) {
    v.resize(n);
    for (size_t k = 0; k < n; k++) in >> v[k];
}

void readPair(std::istream& in, PairForce& f, int n, int stride, bool dispersion) {
    int useSwitch;
    in >> f.method >> f.cutoff >> useSwitch >> f.switchDist >> f.softcore >> f.group;
    f.useSwitch = useSwitch != 0;
    if (dispersion) {
        int lrc;
        in >> f.damping >> lrc;
        f.lrc = lrc != 0;
    }
    else in >> f.overlap;
    f.stride = stride;
    readVec(in, f.params, (size_t)stride * n);
    readVec(in, f.alch, n);
    int ne;
    in >> ne;
    readVec(in, f.excl, 2 * (size_t)ne);
}

int main(int argc, char** argv) {
    if (argc != 3) {
        std::cerr << "usage: kernels_from_file <input> <output>\n";
        return 2;
    }
    std::ifstream in(argv[1]);
    System system;
    ArrayContext context;
    in >> system.n;
    for (double& b : context.box) in >> b;
    in >> context.lambda;
    readVec(in, context.pos, 3 * (size_t)system.n);
    context.forces.assign(3 * (size_t)system.n, 0.0);
    PairForce disp, exch, sr;
    readPair(in, disp, system.n, 5, true);
    readPair(in, exch, system.n, 2, false);
    readPair(in, sr, system.n, 3, false);
    ThreeBodyForce atm;
    int ns, periodic;
    in >> ns >> atm.cutoff >> atm.scale >> atm.dampingMethod >> atm.damping >> atm.centroid >> periodic >> atm.group;
    atm.periodic = periodic != 0;
    for (int s = 0; s < ns; s++) {
        int k;
        in >> k;
        std::vector<int> p(k);
        for (int& q : p) in >> q;
        atm.particles.push_back(p);
        double a, f, w;
        int mol, al;
        in >> a >> f >> w >> mol >> al;
        atm.params.insert(atm.params.end(), {a, f, w});
        atm.molecule.push_back(mol);
        atm.alch.push_back(al);
    }
    try {
        auto shared = std::make_shared<InteraxB200::SharedContext>(system.n, 0, context.box);
        std::vector<std::unique_ptr<InteraxB200::KernelBase>> kernels;
        for (const char* name : {"CalcInteraxDispersionForce", "CalcInteraxExchangeForce", "CalcInteraxShortRangeForce",
                                 "CalcInteraxThreeBodyForce"})
            kernels.push_back(InteraxB200::createKernel(name, shared));
        static_cast<InteraxB200::B200CalcInteraxDispersionForceKernel&>(*kernels[0]).initialize(system, disp);
        static_cast<InteraxB200::B200CalcInteraxExchangeForceKernel&>(*kernels[1]).initialize(system, exch);
        static_cast<InteraxB200::B200CalcInteraxShortRangeForceKernel&>(*kernels[2]).initialize(system, sr);
        if (ns > 0) static_cast<InteraxB200::B200CalcInteraxThreeBodyForceKernel&>(*kernels[3]).initialize(system, atm);
        context.id = 1;
        double e[4];
        for (int k = 0; k < 4; k++) e[k] = (k < 3 || ns > 0) ? kernels[k]->execute(context, true, true) : 0.0;
        std::ofstream out(argv[2]);
        out.precision(17);
        out << e[0] << " " << e[1] << " " << e[2] << " " << e[3] << "\n";
        for (double f : context.forces) out << f << "\n";
        // the factory rejects names this platform does not provide, with the reference's message
        try {
            InteraxB200::createKernel("CalcInteraxMultipoleForce", shared);
            out << "factory: accepted\n";
        }
        catch (const InteraxB200::Exception& ex) {
            out << "factory: " << ex.what() << "\n";
        }
    }
    catch (const InteraxB200::Exception& ex) {
        std::cerr << "error: " << ex.what() << "\n";
        return 1;
    }
    return 0;
}
