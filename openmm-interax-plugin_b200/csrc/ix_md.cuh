// Velocity-Verlet integration on the device (units nm, ps, amu, kJ/mol: a = F/m in nm/ps^2).
#pragma once

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

}  // namespace ix
