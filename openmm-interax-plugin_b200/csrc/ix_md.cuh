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
// cluster of constrained particles by one thread.  Positions: the SHAKE equations (J.-P. Ryckaert, G. Ciccotti and
// H. J. C. Berendsen, J. Comput. Phys. 23, 327 (1977): each particle moved along the cluster's bonds before the
// drift) solved for all the cluster's multipliers at once by Newton's method, as in M-SHAKE (A. Kraeutler, W. F. van
// Gunsteren and P. H. Huenenberger, J. Comput. Chem. 22, 501 (2001)), which converges quadratically where a sweep
// over the constraints one by one converges slowly for coupled bonds.  Velocities: the second stage of RATTLE
// (H. C. Andersen, J. Comput. Phys. 52, 24 (1983)), whose conditions are linear in the multipliers, solved in one step
// with one refinement.  A particle without constraints is a cluster of one, so the cluster kernels move every particle.
constexpr int kMaxClusterParticles = 8;
constexpr int kMaxClusterConstraints = 12;
// one thread per cluster in blocks of one warp: a few thousand clusters still spread over every SM
constexpr int kClusterBlock = 32;

// Solve the n x n system a x = b in place (b becomes x) by Gaussian elimination with partial pivoting; a row-major
// with a leading dimension of kMaxClusterConstraints.  Returns false for a singular matrix.
__device__ __forceinline__ bool solveSmall(double (&a)[kMaxClusterConstraints][kMaxClusterConstraints],
                                           double (&b)[kMaxClusterConstraints], int n) {
    for (int col = 0; col < n; col++) {
        int piv = col;
        for (int r = col + 1; r < n; r++)
            if (fabs(a[r][col]) > fabs(a[piv][col])) piv = r;
        if (a[piv][col] == 0.0) return false;
        if (piv != col) {
            for (int k = 0; k < n; k++) {
                const double t = a[col][k];
                a[col][k] = a[piv][k];
                a[piv][k] = t;
            }
            const double t = b[col];
            b[col] = b[piv];
            b[piv] = t;
        }
        const double inv = 1.0 / a[col][col];
        for (int r = col + 1; r < n; r++) {
            const double f = a[r][col] * inv;
            if (f == 0.0) continue;
            for (int k = col; k < n; k++) a[r][k] -= f * a[col][k];
            b[r] -= f * b[col];
        }
    }
    for (int r = n - 1; r >= 0; r--) {
        double sum = b[r];
        for (int k = r + 1; k < n; k++) sum -= a[r][k] * b[k];
        b[r] = sum / a[r][r];
    }
    return true;
}

// The coupling of constraint l's multiplier to constraint k's bond: how the bond vector of k changes per unit of l's
// multiplier, as the coefficient of l's direction (w_p for the first particle of l, -w_q for its second).
__device__ __forceinline__ double constraintCoupling(int2 k, int2 l, const double* w) {
    const double ap = (k.x == l.x ? w[k.x] : 0.0) - (k.x == l.y ? w[k.x] : 0.0);
    const double aq = (k.y == l.x ? w[k.y] : 0.0) - (k.y == l.y ? w[k.y] : 0.0);
    return ap - aq;
}

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

// A rigid triangle (a 3-site water): 3 particles and the constraints (0,1), (0,2), (1,2) in this order, which the host
// arranges.  Its solves take every index at compile time, so the cluster stays in registers.
__device__ __forceinline__ int2 triPair(int q) { return make_int2(q == 2 ? 1 : 0, q == 0 ? 1 : 2); }

__device__ __forceinline__ bool isTriangle(const ConstraintClusters& K, int c0, int np, int nc) {
    if (np != 3 || nc != 3) return false;
    const int2 a = K.pair[c0], b = K.pair[c0 + 1], c = K.pair[c0 + 2];
    return a.x == 0 && a.y == 1 && b.x == 0 && b.y == 2 && c.x == 1 && c.y == 2;
}

// Solve the 3 x 3 system a x = b by the adjugate (Cramer's rule); false for a singular matrix.
__device__ __forceinline__ bool solve3(const double (&a)[3][3], double (&b)[3]) {
    const double i00 = a[1][1] * a[2][2] - a[1][2] * a[2][1], i01 = a[0][2] * a[2][1] - a[0][1] * a[2][2],
                 i02 = a[0][1] * a[1][2] - a[0][2] * a[1][1];
    const double i10 = a[1][2] * a[2][0] - a[1][0] * a[2][2], i11 = a[0][0] * a[2][2] - a[0][2] * a[2][0],
                 i12 = a[0][2] * a[1][0] - a[0][0] * a[1][2];
    const double i20 = a[1][0] * a[2][1] - a[1][1] * a[2][0], i21 = a[0][1] * a[2][0] - a[0][0] * a[2][1],
                 i22 = a[0][0] * a[1][1] - a[0][1] * a[1][0];
    const double det = a[0][0] * i00 + a[0][1] * i10 + a[0][2] * i20;
    if (det == 0.0) return false;
    const double inv = 1.0 / det;
    const double x0 = (i00 * b[0] + i01 * b[1] + i02 * b[2]) * inv;
    const double x1 = (i10 * b[0] + i11 * b[1] + i12 * b[2]) * inv;
    const double x2 = (i20 * b[0] + i21 * b[1] + i22 * b[2]) * inv;
    b[0] = x0;
    b[1] = x1;
    b[2] = x2;
    return true;
}

// One cluster of kConstrainedDrift; returns whether one of its particles moved more than the list allows.  TRI: the
// cluster is a rigid triangle (isTriangle).
template <bool TRI>
__device__ __forceinline__ bool constrainedDriftCluster(ConstraintClusters K, int c, double dt, const double* invMass,
                                                        const double* force, double* vel, double* pos,
                                                        const ListBuffers& L, bool refresh, float maxMove2) {
    constexpr int MP = TRI ? 3 : kMaxClusterParticles, MC = TRI ? 3 : kMaxClusterConstraints;
    constexpr int kUnroll = TRI ? 3 : 1;   // the general cluster keeps its loops (and arrays in local memory)
    const int p0 = K.particleStart[c], np = TRI ? 3 : K.particleStart[c + 1] - p0;
    const int c0 = K.constraintStart[c], nc = TRI ? 3 : K.constraintStart[c + 1] - c0;
    const double h = 0.5 * dt;
    bool moved = false;
    double old[MP][3], x[MP][3], w[MP];
#pragma unroll kUnroll
    for (int k = 0; k < MP; k++) {
        if (k >= np) break;
        const int i = K.particles[p0 + k];
        w[k] = invMass[i];
#pragma unroll kUnroll
        for (int d = 0; d < 3; d++) {
            old[k][d] = pos[3 * i + d];
            x[k][d] = old[k][d] + dt * (vel[3 * i + d] + h * w[k] * force[3 * i + d]);
        }
    }
    // Newton on g_k(lambda) = d_k^2 - |s_k|^2 = 0, s_k the bond of constraint k, each particle moved along the
    // pre-drift bonds r_l: x_p += w_p lambda_l r_l, x_q -= w_q lambda_l r_l
    int2 pair[MC];
    double r0[MC][3], d2[MC];
#pragma unroll kUnroll
    for (int q = 0; q < MC; q++) {
        if (q >= nc) break;
        pair[q] = TRI ? triPair(q) : K.pair[c0 + q];
        d2[q] = K.dist2[c0 + q];
#pragma unroll kUnroll
        for (int d = 0; d < 3; d++) r0[q][d] = old[pair[q].x][d] - old[pair[q].y][d];
    }
    bool converged = false;
    for (int iteration = 0; iteration < 30; iteration++) {
        double s[MC][3], g[MC];
        double worst = 0.0;
#pragma unroll kUnroll
        for (int k = 0; k < MC; k++) {
            if (k >= nc) break;
#pragma unroll kUnroll
            for (int d = 0; d < 3; d++) s[k][d] = x[pair[k].x][d] - x[pair[k].y][d];
            g[k] = d2[k] - (s[k][0] * s[k][0] + s[k][1] * s[k][1] + s[k][2] * s[k][2]);
            worst = fmax(worst, fabs(g[k]) / d2[k]);
        }
        if (worst <= K.tolerance) {
            converged = true;
            break;
        }
        double J[MC][MC];
#pragma unroll kUnroll
        for (int k = 0; k < MC; k++) {
            if (k >= nc) break;
#pragma unroll kUnroll
            for (int l = 0; l < MC; l++) {
                if (l >= nc) break;
                const double cp = constraintCoupling(pair[k], pair[l], w);
                J[k][l] = cp == 0.0 ? 0.0 : 2.0 * cp * (s[k][0] * r0[l][0] + s[k][1] * r0[l][1] + s[k][2] * r0[l][2]);
            }
        }
        bool solved;
        if constexpr (TRI) solved = solve3(J, g);
        else solved = solveSmall(J, g, nc);
        if (!solved) break;
#pragma unroll kUnroll
        for (int l = 0; l < MC; l++) {
            if (l >= nc) break;
#pragma unroll kUnroll
            for (int d = 0; d < 3; d++) {
                x[pair[l].x][d] += g[l] * w[pair[l].x] * r0[l][d];
                x[pair[l].y][d] -= g[l] * w[pair[l].y] * r0[l][d];
            }
        }
    }
    if (!converged) atomicOr(K.fail, 1);
    const double invDt = 1.0 / dt;
#pragma unroll kUnroll
    for (int k = 0; k < MP; k++) {
        if (k >= np) break;
        const int i = K.particles[p0 + k];
#pragma unroll kUnroll
        for (int d = 0; d < 3; d++) {
            vel[3 * i + d] = (x[k][d] - old[k][d]) * invDt;
            pos[3 * i + d] = x[k][d];
        }
        if (refresh) moved |= refreshSlot(L, i, x[k], maxMove2);
    }
    return moved;
}

// A cluster without constraints (a single particle): half kick and drift.
__device__ __forceinline__ bool freeDriftCluster(ConstraintClusters K, int c, double dt, const double* invMass,
                                                 const double* force, double* vel, double* pos, const ListBuffers& L,
                                                 bool refresh, float maxMove2) {
    const int p0 = K.particleStart[c], np = K.particleStart[c + 1] - p0;
    const double h = 0.5 * dt;
    bool moved = false;
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

// First half kick and drift of every particle, then SHAKE: the constrained particles of each cluster are moved along
// the bonds of the positions before the drift until every distance is met (Newton on all of the cluster's
// multipliers, at most 30 iterations; quadratic convergence takes 3 to 4 from a 1 fs drift); their velocities become
// the constrained displacement over dt.  With `refresh` (a pair list exists) the new positions also go to the list's sorted slots,
// and a particle that moved more than the list allows requests a rebuild.
__global__ void kConstrainedDrift(ConstraintClusters K, double dt, const double* invMass, const double* force,
                                  double* vel, double* pos, ListBuffers L, bool refresh, float maxMove2) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    bool moved = false;
    if (c < K.num) {
        const int c0 = K.constraintStart[c], nc = K.constraintStart[c + 1] - c0;
        const int np = K.particleStart[c + 1] - K.particleStart[c];
        if (nc == 0) moved = freeDriftCluster(K, c, dt, invMass, force, vel, pos, L, refresh, maxMove2);
        else if (isTriangle(K, c0, np, nc))
            moved = constrainedDriftCluster<true>(K, c, dt, invMass, force, vel, pos, L, refresh, maxMove2);
        else moved = constrainedDriftCluster<false>(K, c, dt, invMass, force, vel, pos, L, refresh, maxMove2);
    }
    if (refresh && __any_sync(0xffffffffu, moved) && (threadIdx.x & 31) == 0) atomicOr(L.flag, 1);
}

// The velocity stage of one constrained cluster (TRI: a rigid triangle, isTriangle).
template <bool TRI>
__device__ __forceinline__ void constrainClusterVelocities(ConstraintClusters K, int c, const double* invMass,
                                                           const double* pos, double* vel) {
    constexpr int MP = TRI ? 3 : kMaxClusterParticles, MC = TRI ? 3 : kMaxClusterConstraints;
    constexpr int kUnroll = TRI ? 3 : 1;   // the general cluster keeps its loops (and arrays in local memory)
    const int p0 = K.particleStart[c], np = TRI ? 3 : K.particleStart[c + 1] - p0;
    const int c0 = K.constraintStart[c], nc = TRI ? 3 : K.constraintStart[c + 1] - c0;
    double x[MP][3], v[MP][3], w[MP];
#pragma unroll kUnroll
    for (int k = 0; k < MP; k++) {
        if (k >= np) break;
        const int i = K.particles[p0 + k];
        w[k] = invMass[i];
#pragma unroll kUnroll
        for (int d = 0; d < 3; d++) {
            x[k][d] = pos[3 * i + d];
            v[k][d] = vel[3 * i + d];
        }
    }
    // conditions r_k . (v_p - v_q) = 0 after v_i += sum_l a_{l,i} mu_l r_l: linear in mu, solved directly, then
    // once more on the residual (rounding)
    int2 pair[MC];
    double r[MC][3];
#pragma unroll kUnroll
    for (int q = 0; q < MC; q++) {
        if (q >= nc) break;
        pair[q] = TRI ? triPair(q) : K.pair[c0 + q];
#pragma unroll kUnroll
        for (int d = 0; d < 3; d++) r[q][d] = x[pair[q].x][d] - x[pair[q].y][d];
    }
    bool converged = false;
    for (int pass = 0; pass < 3; pass++) {
        double rhs[MC];
        double worst = 0.0;
#pragma unroll kUnroll
        for (int k = 0; k < MC; k++) {
            if (k >= nc) break;
            const double r2 = r[k][0] * r[k][0] + r[k][1] * r[k][1] + r[k][2] * r[k][2];
            double dot = 0.0;
#pragma unroll kUnroll
            for (int d = 0; d < 3; d++) dot += r[k][d] * (v[pair[k].x][d] - v[pair[k].y][d]);
            rhs[k] = -dot;
            worst = fmax(worst, fabs(dot) / r2);    // stretching rate per ps
        }
        if (worst <= K.tolerance) {
            converged = true;
            break;
        }
        double M[MC][MC];
#pragma unroll kUnroll
        for (int k = 0; k < MC; k++) {
            if (k >= nc) break;
#pragma unroll kUnroll
            for (int l = 0; l < MC; l++) {
                if (l >= nc) break;
                const double cp = constraintCoupling(pair[k], pair[l], w);
                M[k][l] = cp == 0.0 ? 0.0 : cp * (r[k][0] * r[l][0] + r[k][1] * r[l][1] + r[k][2] * r[l][2]);
            }
        }
        bool solved;
        if constexpr (TRI) solved = solve3(M, rhs);
        else solved = solveSmall(M, rhs, nc);
        if (!solved) break;
#pragma unroll kUnroll
        for (int l = 0; l < MC; l++) {
            if (l >= nc) break;
#pragma unroll kUnroll
            for (int d = 0; d < 3; d++) {
                v[pair[l].x][d] += rhs[l] * w[pair[l].x] * r[l][d];
                v[pair[l].y][d] -= rhs[l] * w[pair[l].y] * r[l][d];
            }
        }
    }
    if (!converged) atomicOr(K.fail, 1);
#pragma unroll kUnroll
    for (int k = 0; k < MP; k++) {
        if (k >= np) break;
        const int i = K.particles[p0 + k];
#pragma unroll kUnroll
        for (int d = 0; d < 3; d++) vel[3 * i + d] = v[k][d];
    }
}

// Velocities of each constrained cluster with the components along its bonds removed (no bond stretches), after the
// second half kick: one linear solve of the cluster's multipliers and at most two refinements of the residual.
__global__ void kConstrainVelocities(ConstraintClusters K, const double* invMass, const double* pos, double* vel) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= K.num) return;
    const int c0 = K.constraintStart[c], nc = K.constraintStart[c + 1] - c0;
    if (nc == 0) return;
    const int np = K.particleStart[c + 1] - K.particleStart[c];
    if (isTriangle(K, c0, np, nc)) constrainClusterVelocities<true>(K, c, invMass, pos, vel);
    else constrainClusterVelocities<false>(K, c, invMass, pos, vel);
}

}  // namespace ix
