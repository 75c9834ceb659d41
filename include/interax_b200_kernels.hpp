/* C++ kernel classes of the InteraxFF short-range path on B200, over the C ABI of interax_b200.h.
 *
 * They replace the reference plugin's platform kernels CalcInteraxDispersionForceKernel, CalcInteraxExchangeForceKernel,
 * CalcInteraxShortRangeForceKernel and CalcInteraxThreeBodyForceKernel (openmmapi/include/InteraxKernels.h:51-189)
 * with the same names (Name()), the same methods (initialize, execute, copyParametersToContext) and the same error
 * messages (thrown as InteraxB200::Exception).  OpenMM is not a dependency: the Force arguments are templates that
 * need only the reference Force classes' accessors (getNumParticles, getParticleParameters, getNonbondedMethod, ...),
 * so OpenMM's own InteraxDispersionForce & co. fit, and the platform's ContextImpl is reached through ContextAccess,
 * which a platform implements in a few lines (positions, box, parameters, where forces go).
 *
 * The three pair forces of a context are evaluated together in one fused pass, so the four kernels of one context
 * share one SharedContext (one ix_ctx): the first kernel executed in an evaluation computes every selected term and
 * adds all their forces; each kernel returns its own term's energy.  createKernel() is the factory keyed by the
 * reference's kernel names.
 */
#ifndef INTERAX_B200_KERNELS_HPP
#define INTERAX_B200_KERNELS_HPP

#include <cstdint>
#include <memory>
#include <set>
#include <stdexcept>
#include <string>
#include <vector>

#include "interax_b200.h"

namespace InteraxB200 {

class Exception : public std::runtime_error {
public:
    using std::runtime_error::runtime_error;
};

/* What the kernels read from and write to the platform's context for one evaluation. */
class ContextAccess {
public:
    virtual ~ContextAccess() = default;
    virtual int getNumParticles() const = 0;
    virtual void getPositions(std::vector<double>& xyz) const = 0;        // n x 3, nm
    virtual void getPeriodicBoxVectors(double box[9]) const = 0;          // a, b, c
    virtual double getParameter(const std::string& name) const = 0;       // context parameters (alchemical lambdas)
    virtual int getEvaluationGroups() const { return -1; }               // force groups of the current evaluation
    virtual long long getEvaluationId() const = 0;                        // differs between evaluations
    virtual void addForces(const std::vector<double>& forces) = 0;        // n x 3, kJ/mol/nm, added
};

/* One ix_ctx per context, shared by the context's four kernels. */
class SharedContext {
public:
    SharedContext(int numParticles, int device, const double defaultBox[9]) {
        if (ix_ctx_create(numParticles, device, defaultBox, &ctx_) != IX_OK) throw Exception(ix_last_error(nullptr));
    }
    ~SharedContext() { ix_ctx_destroy(ctx_); }
    SharedContext(const SharedContext&) = delete;
    SharedContext& operator=(const SharedContext&) = delete;

    ix_ctx* get() const { return ctx_; }
    void check(int rc) const {
        if (rc != IX_OK) throw Exception(ix_last_error(ctx_));
    }
    void addParameterName(const std::string& name) { parameters_.insert(name); }
    void invalidate() { lastId_ = -1; }

    /* The energy of one term (0 dispersion, 1 exchange, 2 short range, 3 three-body) of the current evaluation. The
     * first call of an evaluation computes every term selected by the evaluation's groups; forces are added once. */
    double energyOf(int term, ContextAccess& context, bool includeForces) {
        const long long id = context.getEvaluationId();
        const int groups = context.getEvaluationGroups();
        if (id != lastId_ || groups != lastGroups_) {
            std::vector<double> xyz;
            context.getPositions(xyz);
            double box[9];
            context.getPeriodicBoxVectors(box);
            for (const std::string& name : parameters_) check(ix_set_parameter(ctx_, name.c_str(), context.getParameter(name)));
            check(ix_set_positions(ctx_, xyz.data(), box));
            forces_.resize(xyz.size());
            double total = 0.0;
            check(ix_compute(ctx_, groups, 1, 1, terms_, &total, forces_.data()));
            lastId_ = id;
            lastGroups_ = groups;
            forcesAdded_ = false;
        }
        if (includeForces && !forcesAdded_) {
            context.addForces(forces_);
            forcesAdded_ = true;
        }
        return terms_[term];
    }

private:
    ix_ctx* ctx_ = nullptr;
    std::set<std::string> parameters_;
    long long lastId_ = -1;
    int lastGroups_ = 0;
    bool forcesAdded_ = false;
    double terms_[4] = {0, 0, 0, 0};
    std::vector<double> forces_;
};

namespace detail {

// The settings every pair force shares (InteraxPairForce), with the storage their pointers refer to.
struct PairSettings {
    std::vector<int32_t> exclusions;
    std::string alchemical;
    ix_pair_settings s{};
    template <class Force>
    explicit PairSettings(const Force& force) : alchemical(force.getAlchemicalParameterName()) {
        const int ne = force.getNumExclusions();
        exclusions.resize(2 * (size_t)ne);
        for (int k = 0; k < ne; k++) {
            int p1, p2;
            force.getExclusionParticles(k, p1, p2);
            exclusions[2 * k] = p1;
            exclusions[2 * k + 1] = p2;
        }
        s.nonbonded_method = (int)force.getNonbondedMethod();
        s.cutoff = force.getCutoffDistance();
        s.use_switching_function = force.getUseSwitchingFunction() ? 1 : 0;
        s.switching_distance = force.getSwitchingDistance();
        s.softcore_radius = force.getSoftcoreRadius();
        s.force_group = force.getForceGroup();
        s.alchemical_parameter = alchemical.c_str();
        s.num_exclusions = ne;
        s.exclusions = exclusions.data();
    }
};

template <class Force>
void checkCount(const Force& force, int numParticles, const char* name) {
    if (force.getNumParticles() != numParticles)
        throw Exception(std::string(name) + " must have exactly as many particles as the System it belongs to.");
}

template <class Force>
std::vector<double> dispersionParams(const Force& f, std::vector<uint8_t>* alch) {
    const int n = f.getNumParticles();
    std::vector<double> p(5 * (size_t)n);
    if (alch) alch->resize(n);
    for (int i = 0; i < n; i++) {
        bool a;
        f.getParticleParameters(i, p[5 * i], p[5 * i + 1], p[5 * i + 2], p[5 * i + 3], p[5 * i + 4], a);
        if (alch) (*alch)[i] = a;
    }
    return p;
}

template <class Force>
std::vector<double> exchangeParams(const Force& f, std::vector<uint8_t>* alch) {
    const int n = f.getNumParticles();
    std::vector<double> p(2 * (size_t)n);
    if (alch) alch->resize(n);
    for (int i = 0; i < n; i++) {
        bool a;
        f.getParticleParameters(i, p[2 * i], p[2 * i + 1], a);
        if (alch) (*alch)[i] = a;
    }
    return p;
}

template <class Force>
std::vector<double> shortRangeParams(const Force& f, std::vector<uint8_t>* alch) {
    const int n = f.getNumParticles();
    std::vector<double> p(3 * (size_t)n);
    if (alch) alch->resize(n);
    for (int i = 0; i < n; i++) {
        bool a;
        f.getParticleParameters(i, p[3 * i], p[3 * i + 1], p[3 * i + 2], a);
        if (alch) (*alch)[i] = a;
    }
    return p;
}

}  // namespace detail

/* Common part of the four kernels: the shared context and the term the kernel returns. */
class KernelBase {
public:
    KernelBase(std::shared_ptr<SharedContext> shared, int term) : shared_(std::move(shared)), term_(term) {}
    virtual ~KernelBase() = default;
    /* Returns the energy of this kernel's force and (through the first kernel of the evaluation) adds the forces of
     * every force selected by the evaluation's groups. */
    double execute(ContextAccess& context, bool includeForces, bool includeEnergy) {
        const double e = shared_->energyOf(term_, context, includeForces);
        return includeEnergy ? e : 0.0;
    }

protected:
    std::shared_ptr<SharedContext> shared_;
    int term_;
};

class B200CalcInteraxDispersionForceKernel : public KernelBase {
public:
    static std::string Name() { return "CalcInteraxDispersionForce"; }
    explicit B200CalcInteraxDispersionForceKernel(std::shared_ptr<SharedContext> shared) : KernelBase(shared, 0) {}
    template <class System, class Force>
    void initialize(const System& system, const Force& force) {
        detail::checkCount(force, system.getNumParticles(), "InteraxDispersionForce");
        detail::PairSettings s(force);
        std::vector<uint8_t> alch;
        const std::vector<double> p = detail::dispersionParams(force, &alch);
        shared_->check(ix_add_dispersion(shared_->get(), &s.s, p.data(), alch.data(), force.getDampingScale(),
                                         force.getUseLongRangeCorrection() ? 1 : 0));
        shared_->addParameterName(force.getAlchemicalParameterName());
        shared_->invalidate();
    }
    template <class Context, class Force>
    void copyParametersToContext(Context&, const Force& force) {
        const std::vector<double> p = detail::dispersionParams(force, nullptr);
        shared_->check(ix_update_dispersion(shared_->get(), p.data(), force.getDampingScale()));
        shared_->invalidate();
    }
};

class B200CalcInteraxExchangeForceKernel : public KernelBase {
public:
    static std::string Name() { return "CalcInteraxExchangeForce"; }
    explicit B200CalcInteraxExchangeForceKernel(std::shared_ptr<SharedContext> shared) : KernelBase(shared, 1) {}
    template <class System, class Force>
    void initialize(const System& system, const Force& force) {
        detail::checkCount(force, system.getNumParticles(), "InteraxExchangeForce");
        detail::PairSettings s(force);
        std::vector<uint8_t> alch;
        const std::vector<double> p = detail::exchangeParams(force, &alch);
        shared_->check(ix_add_exchange(shared_->get(), &s.s, p.data(), alch.data(), (int)force.getOverlapMethod()));
        shared_->addParameterName(force.getAlchemicalParameterName());
        shared_->invalidate();
    }
    template <class Context, class Force>
    void copyParametersToContext(Context&, const Force& force) {
        const std::vector<double> p = detail::exchangeParams(force, nullptr);
        shared_->check(ix_update_exchange(shared_->get(), p.data(), (int)force.getOverlapMethod()));
        shared_->invalidate();
    }
};

class B200CalcInteraxShortRangeForceKernel : public KernelBase {
public:
    static std::string Name() { return "CalcInteraxShortRangeForce"; }
    explicit B200CalcInteraxShortRangeForceKernel(std::shared_ptr<SharedContext> shared) : KernelBase(shared, 2) {}
    template <class System, class Force>
    void initialize(const System& system, const Force& force) {
        detail::checkCount(force, system.getNumParticles(), "InteraxShortRangeForce");
        detail::PairSettings s(force);
        std::vector<uint8_t> alch;
        const std::vector<double> p = detail::shortRangeParams(force, &alch);
        shared_->check(ix_add_short_range(shared_->get(), &s.s, p.data(), alch.data(), (int)force.getOverlapMethod()));
        shared_->addParameterName(force.getAlchemicalParameterName());
        shared_->invalidate();
    }
    template <class Context, class Force>
    void copyParametersToContext(Context&, const Force& force) {
        const std::vector<double> p = detail::shortRangeParams(force, nullptr);
        shared_->check(ix_update_short_range(shared_->get(), p.data(), (int)force.getOverlapMethod()));
        shared_->invalidate();
    }
};

namespace detail {

struct Sites {
    std::vector<int32_t> offsets{0}, particles, molecule;
    std::vector<double> params;
    std::vector<uint8_t> alch;
    template <class Force>
    explicit Sites(const Force& f) {
        for (int s = 0; s < f.getNumSites(); s++) {
            std::vector<int> part;
            double alpha, frequency, width;
            int mol;
            bool a;
            f.getSiteParameters(s, part, alpha, frequency, width, mol, a);
            particles.insert(particles.end(), part.begin(), part.end());
            offsets.push_back((int32_t)particles.size());
            params.insert(params.end(), {alpha, frequency, width});
            molecule.push_back(mol);
            alch.push_back(a ? 1 : 0);
        }
    }
};

}  // namespace detail

class B200CalcInteraxThreeBodyForceKernel : public KernelBase {
public:
    static std::string Name() { return "CalcInteraxThreeBodyForce"; }
    explicit B200CalcInteraxThreeBodyForceKernel(std::shared_ptr<SharedContext> shared) : KernelBase(shared, 3) {}
    template <class System, class Force>
    void initialize(const System&, const Force& force) {
        detail::Sites s(force);
        const std::string alch = force.getAlchemicalParameterName();
        shared_->check(ix_add_three_body(shared_->get(), force.getNumSites(), s.offsets.data(), s.particles.data(),
                                         s.params.data(), s.molecule.data(), s.alch.data(), force.getCutoffDistance(),
                                         force.getScaleFactor(), (int)force.getDampingMethod(),
                                         force.getDampingScale(), force.getCentroidDampingRadius(),
                                         force.usesPeriodicBoundaryConditions() ? 1 : 0, alch.c_str(),
                                         force.getForceGroup()));
        shared_->addParameterName(alch);
        shared_->invalidate();
    }
    template <class Context, class Force>
    void copyParametersToContext(Context&, const Force& force) {
        detail::Sites s(force);
        shared_->check(ix_update_three_body(shared_->get(), s.params.data(), force.getScaleFactor(),
                                            force.getDampingScale(), force.getCentroidDampingRadius()));
        shared_->invalidate();
    }
};

/* The kernel factory, keyed by the reference's kernel names (its CudaInteraxKernelFactory::createKernelImpl,
 * platforms/cuda/src/CudaInteraxKernelFactory.cpp:74-87).  The kernels of one context share `shared`. */
inline std::unique_ptr<KernelBase> createKernel(const std::string& name, std::shared_ptr<SharedContext> shared) {
    if (name == B200CalcInteraxDispersionForceKernel::Name())
        return std::unique_ptr<KernelBase>(new B200CalcInteraxDispersionForceKernel(shared));
    if (name == B200CalcInteraxExchangeForceKernel::Name())
        return std::unique_ptr<KernelBase>(new B200CalcInteraxExchangeForceKernel(shared));
    if (name == B200CalcInteraxShortRangeForceKernel::Name())
        return std::unique_ptr<KernelBase>(new B200CalcInteraxShortRangeForceKernel(shared));
    if (name == B200CalcInteraxThreeBodyForceKernel::Name())
        return std::unique_ptr<KernelBase>(new B200CalcInteraxThreeBodyForceKernel(shared));
    throw Exception("Tried to create kernel with illegal kernel name '" + name + "'");
}

}  // namespace InteraxB200

#endif /* INTERAX_B200_KERNELS_HPP */
