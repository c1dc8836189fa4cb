// C++ host over the C ABI: the adapter a reference maintainer adds
// (PrimalDualGpuForceSolver, a ForceSolver whose fillForces forwards to
// pdc_solve; reference interface src/Solver/ForceSolverBase.h:78-82), run on
// reference-shaped records.  Stand-ins with the reference's field names replace
// RigidObjectBase (pose, velocities, mass, principal inertia, static flag and
// the acceleration()/angularAcc() outputs) and ContactInformation (objId, pos,
// frame, depth, localForce; src/Contact/ContactInfo.h:12-144).
//
//   force_solver_host <input.bin> <output.bin> [iterations] [tolerance]
//
// input.bin: int32 nb, nc; per body: pos[3] quat[4 xyzw] vel[3] ang[3] mass
// I0[3] (float64) static (uint8); per contact: objId[2] (int32) pos[3]
// frame[9] depth (float64).  output.bin: int32 status, newton_iters; per body
// dv[3] dw[3]; per contact localForce[3] (float64).
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <stdexcept>
#include <string>
#include <vector>

#include "pdc.h"

struct RigidObject {
    double translation[3], rotation[4];  // quaternion x y z w
    double velocity[3], angularVel[3];
    double mass, inertia0[3];
    bool isStatic;
    double acceleration[3], angularAcc[3];  // velocity increments written by the solver
};

struct ContactInformation {
    int objId[2];
    double pos[3];
    double frame[9];  // R: columns normal, t1, t2 (top 3x3 of transformation[0])
    double depth;
    double localForce[3];
};

static void rotation_matrix(const double* q, double* R) {
    const double x = q[0], y = q[1], z = q[2], w = q[3];
    R[0] = 1 - 2 * (y * y + z * z); R[1] = 2 * (x * y - z * w);     R[2] = 2 * (x * z + y * w);
    R[3] = 2 * (x * y + z * w);     R[4] = 1 - 2 * (x * x + z * z); R[5] = 2 * (y * z - x * w);
    R[6] = 2 * (x * z - y * w);     R[7] = 2 * (y * z + x * w);     R[8] = 1 - 2 * (x * x + y * y);
}

// R diag(d) R^T as (xx, yy, zz, xy, xz, yz): the rotational block of
// genMassMat / invGenMassMat (RigidObjectBase.cpp:106-119)
static void world_inertia(const double* R, const double* d, double* out) {
    auto e = [&](int i, int j) {
        return R[3 * i] * d[0] * R[3 * j] + R[3 * i + 1] * d[1] * R[3 * j + 1] + R[3 * i + 2] * d[2] * R[3 * j + 2];
    };
    out[0] = e(0, 0); out[1] = e(1, 1); out[2] = e(2, 2);
    out[3] = e(0, 1); out[4] = e(0, 2); out[5] = e(1, 2);
}

class PrimalDualGpuForceSolver {
   public:
    PrimalDualGpuForceSolver(int iterations, double tolerance) {
        pdc_config_default(&cfg_);
        cfg_.max_iter = iterations;
        cfg_.tol = tolerance;
        if (pdc_create(&cfg_, &solver_) != PDC_OK) throw std::runtime_error(pdc_last_error(nullptr));
    }
    ~PrimalDualGpuForceSolver() { pdc_destroy(solver_); }

    // ForceSolver::fillForces: pack SoA, solve, write back the reference's side effects
    pdc_stats fillForces(double dt, const double g[3], std::vector<ContactInformation>& contacts,
                         std::vector<RigidObject>& objects) {
        const int nb = (int)objects.size(), nc = (int)contacts.size();
        vel_.resize(3 * nb); ang_.resize(3 * nb); mass_.resize(nb);
        I_.resize(6 * nb); Ii_.resize(6 * nb); static_.resize(nb);
        for (int b = 0; b < nb; ++b) {
            const RigidObject& o = objects[b];
            double R[9], inv0[3] = {1 / o.inertia0[0], 1 / o.inertia0[1], 1 / o.inertia0[2]};
            rotation_matrix(o.rotation, R);
            for (int k = 0; k < 3; ++k) { vel_[3 * b + k] = o.velocity[k]; ang_[3 * b + k] = o.angularVel[k]; }
            mass_[b] = o.mass;
            world_inertia(R, o.inertia0, &I_[6 * b]);
            world_inertia(R, inv0, &Ii_[6 * b]);
            static_[b] = o.isStatic ? 1 : 0;
        }
        body_.resize(2 * nc); frame_.resize(9 * nc); arm_.resize(6 * nc); depth_.resize(nc);
        for (int i = 0; i < nc; ++i) {
            const ContactInformation& ci = contacts[i];
            for (int j = 0; j < 2; ++j) {
                body_[2 * i + j] = ci.objId[j];
                for (int k = 0; k < 3; ++k) arm_[6 * i + 3 * j + k] = ci.pos[k] - objects[ci.objId[j]].translation[k];
            }
            for (int k = 0; k < 9; ++k) frame_[9 * i + k] = ci.frame[k];
            depth_[i] = ci.depth;
        }
        pdc_bodies_soa B{nb, vel_.data(), ang_.data(), mass_.data(), I_.data(), Ii_.data(), static_.data()};
        pdc_contacts_soa C{nc, body_.data(), frame_.data(), arm_.data(), depth_.data(), nullptr};
        dv_.resize(3 * nb); dw_.resize(3 * nb); f_.resize(3 * nc);
        pdc_result out{dv_.data(), dw_.data(), f_.data(), {}};
        if (pdc_solve(solver_, dt, g, &B, &C, &out) != PDC_OK) throw std::runtime_error(pdc_last_error(solver_));
        for (int b = 0; b < nb; ++b)
            for (int k = 0; k < 3; ++k) {
                objects[b].acceleration[k] = dv_[3 * b + k];
                objects[b].angularAcc[k] = dw_[3 * b + k];
            }
        for (int i = 0; i < nc; ++i)
            for (int k = 0; k < 3; ++k) contacts[i].localForce[k] = f_[3 * i + k];
        return out.stats;
    }

   private:
    pdc_config cfg_;
    pdc_solver* solver_ = nullptr;
    std::vector<double> vel_, ang_, mass_, I_, Ii_, frame_, arm_, depth_, dv_, dw_, f_;
    std::vector<int32_t> body_;
    std::vector<uint8_t> static_;
};

template <class T>
static void rd(FILE* f, T* p, size_t n) {
    if (fread(p, sizeof(T), n, f) != n) throw std::runtime_error("short input file");
}
template <class T>
static void wr(FILE* f, const T* p, size_t n) {
    if (fwrite(p, sizeof(T), n, f) != n) throw std::runtime_error("write failed");
}

int main(int argc, char** argv) {
    if (argc < 3) {
        std::fprintf(stderr, "usage: %s <input.bin> <output.bin> [iterations] [tolerance]\n", argv[0]);
        return 2;
    }
    try {
        FILE* in = std::fopen(argv[1], "rb");
        if (!in) throw std::runtime_error(std::string("cannot open ") + argv[1]);
        int32_t nb, nc;
        double dt, g[3];
        rd(in, &nb, 1); rd(in, &nc, 1); rd(in, &dt, 1); rd(in, g, 3);
        std::vector<RigidObject> objects(nb);
        for (auto& o : objects) {
            rd(in, o.translation, 3); rd(in, o.rotation, 4); rd(in, o.velocity, 3); rd(in, o.angularVel, 3);
            rd(in, &o.mass, 1); rd(in, o.inertia0, 3);
            uint8_t s; rd(in, &s, 1); o.isStatic = s != 0;
        }
        std::vector<ContactInformation> contacts(nc);
        for (auto& c : contacts) {
            int32_t ids[2]; rd(in, ids, 2); c.objId[0] = ids[0]; c.objId[1] = ids[1];
            rd(in, c.pos, 3); rd(in, c.frame, 9); rd(in, &c.depth, 1);
        }
        std::fclose(in);
        PrimalDualGpuForceSolver solver(argc > 3 ? std::atoi(argv[3]) : 100, argc > 4 ? std::atof(argv[4]) : 1e-6);
        const pdc_stats st = solver.fillForces(dt, g, contacts, objects);
        FILE* out = std::fopen(argv[2], "wb");
        if (!out) throw std::runtime_error(std::string("cannot open ") + argv[2]);
        const int32_t head[2] = {st.status, st.newton_iters};
        wr(out, head, 2);
        for (const auto& o : objects) { wr(out, o.acceleration, 3); wr(out, o.angularAcc, 3); }
        for (const auto& c : contacts) wr(out, c.localForce, 3);
        std::fclose(out);
        std::printf("status %d newton_iters %d\n", st.status, st.newton_iters);
    } catch (const std::exception& e) {
        std::fprintf(stderr, "error: %s\n", e.what());
        return 1;
    }
    return 0;
}
