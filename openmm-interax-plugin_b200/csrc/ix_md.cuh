// Velocity-Verlet integration on the device (units nm, ps, amu, kJ/mol: a = F/m in nm/ps^2).
#pragma once

#include "ix_nblist.cuh"

namespace ix {

// v += dt/2 F/m; x += dt v
__global__ void kVerletFirstHalf(int n, double dt, const double* invMass, const double* force, double* vel,
                                 double* pos) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double h = 0.5 * dt * invMass[i];
    for (int d = 0; d < 3; d++) {
        double v = vel[3 * i + d] + h * force[3 * i + d];
        vel[3 * i + d] = v;
        pos[3 * i + d] += dt * v;
    }
}

// v += dt/2 F/m with the new forces
__global__ void kVerletSecondHalf(int n, double dt, const double* invMass, const double* force, double* vel) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double h = 0.5 * dt * invMass[i];
    for (int d = 0; d < 3; d++) vel[3 * i + d] += h * force[3 * i + d];
}

// Distance constraints (OpenMM's System::addConstraint; the benchmark's rigid 3-site waters), solved per connected
// cluster of constrained particles by one thread: positions by SHAKE (J.-P. Ryckaert, G. Ciccotti and H. J. C.
// Berendsen, J. Comput. Phys. 23, 327 (1977)), velocities by the second stage of RATTLE (H. C. Andersen, J. Comput.
// Phys. 52, 24 (1983)), both iterated over the cluster's constraints until every one holds to the tolerance.  A
// particle without constraints is a cluster of one, so the cluster kernels move every particle.
constexpr int kMaxClusterParticles = 8;

struct ConstraintClusters {
    int num;                     // clusters, including the single particles
    const int* particleStart;    // num + 1: the cluster's particles in `particles`
    const int* particles;
    const int* constraintStart;  // num + 1: the cluster's constraints
    const int2* pair;            // the constrained particles, as positions within the cluster
    const double* dist2;         // squared distances
    double tolerance;            // relative, on |r|^2 against d^2 and on the bond's stretching rate
    int* fail;                   // set when a cluster did not converge
};

// A particle's new position into the pair list's sorted slots (the list's build frame), with the displacement check
// that requests a rebuild: the work kStepStart does for an unconstrained step.  Returns whether it moved too far.
__device__ __forceinline__ bool refreshSlot(const ListBuffers& L, int i, const double x[3], float maxMove2) {
    const int s = L.slotOf[i];
    const double sx = x[0] - L.shift[3 * s], sy = x[1] - L.shift[3 * s + 1], sz = x[2] - L.shift[3 * s + 2];
    L.spos[3 * s] = sx;
    L.spos[3 * s + 1] = sy;
    L.spos[3 * s + 2] = sz;
    L.sposf[s] = make_float4((float)sx, (float)sy, (float)sz, 0.0f);
    const double dx = x[0] - L.refPos[3 * i], dy = x[1] - L.refPos[3 * i + 1], dz = x[2] - L.refPos[3 * i + 2];
    return (float)(dx * dx + dy * dy + dz * dz) > maxMove2;
}

// One cluster of kConstrainedDrift; returns whether one of its particles moved more than the list allows.
__device__ __forceinline__ bool constrainedDriftCluster(ConstraintClusters K, int c, double dt, const double* invMass,
                                                        const double* force, double* vel, double* pos,
                                                        const ListBuffers& L, bool refresh, float maxMove2) {
    const int p0 = K.particleStart[c], np = K.particleStart[c + 1] - p0;
    const int c0 = K.constraintStart[c], nc = K.constraintStart[c + 1] - c0;
    const double h = 0.5 * dt;
    bool moved = false;
    if (nc == 0) {
        for (int k = 0; k < np; k++) {
            const int i = K.particles[p0 + k];
            double x[3];
            for (int d = 0; d < 3; d++) {
                const double v = vel[3 * i + d] + h * invMass[i] * force[3 * i + d];
                vel[3 * i + d] = v;
                x[d] = pos[3 * i + d] + dt * v;
                pos[3 * i + d] = x[d];
            }
            if (refresh) moved |= refreshSlot(L, i, x, maxMove2);
        }
        return moved;
    }
    double old[kMaxClusterParticles][3], x[kMaxClusterParticles][3], w[kMaxClusterParticles];
    for (int k = 0; k < np; k++) {
        const int i = K.particles[p0 + k];
        w[k] = invMass[i];
        for (int d = 0; d < 3; d++) {
            old[k][d] = pos[3 * i + d];
            x[k][d] = old[k][d] + dt * (vel[3 * i + d] + h * w[k] * force[3 * i + d]);
        }
    }
    bool converged = false;
    for (int iteration = 0; iteration < 1000 && !converged; iteration++) {
        converged = true;
        for (int q = 0; q < nc; q++) {
            const int2 pq = K.pair[c0 + q];
            const double d2 = K.dist2[c0 + q];
            double s[3], r[3];
            for (int d = 0; d < 3; d++) {
                s[d] = x[pq.x][d] - x[pq.y][d];
                r[d] = old[pq.x][d] - old[pq.y][d];
            }
            const double diff = d2 - (s[0] * s[0] + s[1] * s[1] + s[2] * s[2]);
            if (fabs(diff) > K.tolerance * d2) converged = false;
            const double denom = 2.0 * (s[0] * r[0] + s[1] * r[1] + s[2] * r[2]) * (w[pq.x] + w[pq.y]);
            if (denom == 0.0) continue;
            const double g = diff / denom;
            for (int d = 0; d < 3; d++) {
                x[pq.x][d] += g * w[pq.x] * r[d];
                x[pq.y][d] -= g * w[pq.y] * r[d];
            }
        }
    }
    if (!converged) atomicOr(K.fail, 1);
    const double invDt = 1.0 / dt;
    for (int k = 0; k < np; k++) {
        const int i = K.particles[p0 + k];
        for (int d = 0; d < 3; d++) {
            vel[3 * i + d] = (x[k][d] - old[k][d]) * invDt;
            pos[3 * i + d] = x[k][d];
        }
        if (refresh) moved |= refreshSlot(L, i, x[k], maxMove2);
    }
    return moved;
}

// First half kick and drift of every particle, then SHAKE: the constrained particles of each cluster are moved along
// the bonds of the positions before the drift until every distance is met; their velocities become the constrained
// displacement over dt.  With `refresh` (a pair list exists) the new positions also go to the list's sorted slots,
// and a particle that moved more than the list allows requests a rebuild.
__global__ void kConstrainedDrift(ConstraintClusters K, double dt, const double* invMass, const double* force,
                                  double* vel, double* pos, ListBuffers L, bool refresh, float maxMove2) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    bool moved = false;
    if (c < K.num) moved = constrainedDriftCluster(K, c, dt, invMass, force, vel, pos, L, refresh, maxMove2);
    if (refresh && __any_sync(0xffffffffu, moved) && (threadIdx.x & 31) == 0) atomicOr(L.flag, 1);
}

// Velocities of each constrained cluster with the components along its bonds removed (no bond stretches), after the
// second half kick.
__global__ void kConstrainVelocities(ConstraintClusters K, const double* invMass, const double* pos, double* vel) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= K.num) return;
    const int p0 = K.particleStart[c], np = K.particleStart[c + 1] - p0;
    const int c0 = K.constraintStart[c], nc = K.constraintStart[c + 1] - c0;
    if (nc == 0) return;
    double x[kMaxClusterParticles][3], v[kMaxClusterParticles][3], w[kMaxClusterParticles];
    for (int k = 0; k < np; k++) {
        const int i = K.particles[p0 + k];
        w[k] = invMass[i];
        for (int d = 0; d < 3; d++) {
            x[k][d] = pos[3 * i + d];
            v[k][d] = vel[3 * i + d];
        }
    }
    bool converged = false;
    for (int iteration = 0; iteration < 1000 && !converged; iteration++) {
        converged = true;
        for (int q = 0; q < nc; q++) {
            const int2 pq = K.pair[c0 + q];
            double r[3], dv[3];
            for (int d = 0; d < 3; d++) {
                r[d] = x[pq.x][d] - x[pq.y][d];
                dv[d] = v[pq.x][d] - v[pq.y][d];
            }
            const double r2 = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
            const double rate = (dv[0] * r[0] + dv[1] * r[1] + dv[2] * r[2]) / r2;   // d|r|/dt / |r|
            if (fabs(rate) > K.tolerance) converged = false;
            const double wsum = w[pq.x] + w[pq.y];
            if (wsum == 0.0) continue;
            const double k = rate / wsum;
            for (int d = 0; d < 3; d++) {
                v[pq.x][d] -= k * w[pq.x] * r[d];
                v[pq.y][d] += k * w[pq.y] * r[d];
            }
        }
    }
    if (!converged) atomicOr(K.fail, 1);
    for (int k = 0; k < np; k++) {
        const int i = K.particles[p0 + k];
        for (int d = 0; d < 3; d++) vel[3 * i + d] = v[k][d];
    }
}

}  // namespace ix
