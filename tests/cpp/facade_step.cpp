// Drives the engine through the C++ facade of include/avbd/avbd.hpp the way
// the reference's scene set-up does (one addParticle / addEnergy call per
// particle and element, simobject/TetMeshObject.cpp:53-97), then steps with
// SimulationExecutor::timeStep().
//
// usage: facade_step <scene.bin> <steps> <out.bin>
// scene.bin: u32 n; n*(3 f64 pos, f64 mass, u8 fixed); u32 nt;
//            nt*(4 u32 idx, f64 lambda, f64 mu, f64 kd, 9 f64 Q, f64 V);
//            f64 dt; u32 iters; f64 rho
// out.bin:   n*3 f64 positions
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "avbd/avbd.hpp"

template <typename T>
static T rd(FILE* f) {
    T v;
    if (fread(&v, sizeof(T), 1, f) != 1) {
        fprintf(stderr, "short read\n");
        exit(2);
    }
    return v;
}

int main(int argc, char** argv) {
    if (argc != 4) return 2;
    FILE* f = fopen(argv[1], "rb");
    if (!f) return 2;
    unsigned n = rd<unsigned>(f);
    Sim::SimulationContext ctx(n, 1, 1u << 24, 16, 16);
    std::vector<unsigned> fixed;
    for (unsigned i = 0; i < n; i++) {
        avbd::Vec3 p{rd<double>(f), rd<double>(f), rd<double>(f)};
        double m = rd<double>(f);
        unsigned char fx = rd<unsigned char>(f);
        unsigned slot = ctx.particles.addParticle(p, m);
        if (fx) ctx.particles.setFixed(slot, true);
    }
    unsigned nt = rd<unsigned>(f);
    for (unsigned t = 0; t < nt; t++) {
        std::array<unsigned, 4> idx{rd<unsigned>(f), rd<unsigned>(f), rd<unsigned>(f), rd<unsigned>(f)};
        double lam = rd<double>(f), mu = rd<double>(f), kd = rd<double>(f);
        avbd::Mat3 Q;
        for (double& q : Q) q = rd<double>(f);
        double V = rd<double>(f);
        ctx.energies.neo_hookean.addEnergy(idx, lam, mu, kd, Q, V);
    }
    ctx.params.dt = rd<double>(f);
    unsigned iters = rd<unsigned>(f);
    double rho = rd<double>(f);
    fclose(f);
    Sim::SimulationExecutor exec(&ctx, iters, rho, 0);
    int steps = atoi(argv[2]);
    try {
        for (int s = 0; s < steps; s++) exec.timeStep();
        std::vector<double> x;
        ctx.particles.positions(x);
        FILE* o = fopen(argv[3], "wb");
        fwrite(x.data(), sizeof(double), x.size(), o);
        fclose(o);
    } catch (const avbd::Error& e) {
        fprintf(stderr, "avbd error %d: %s\n", e.code, e.what());
        return 1;
    }
    return 0;
}
