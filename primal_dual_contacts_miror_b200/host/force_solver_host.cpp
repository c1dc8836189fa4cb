// C++ host over the C ABI: the adapter a reference maintainer adds
// (PrimalDualGpuForceSolver, a ForceSolver whose fillForces forwards to
// pdc_solve; reference interface src/Solver/ForceSolverBase.h:78-82), run on
// reference-shaped records.  Stand-ins with the reference's field names replace
// RigidObjectBase (pose, velocities, mass, principal inertia, static flag and
// the acceleration()/angularAcc() outputs) and ContactInformation (objId, pos,
// frame, depth, localForce; src/Contact/ContactInfo.h:12-144).
//
//   force_solver_host <input.bin> <output.bin> [iterations] [tolerance]
//   force_solver_host --solver-yaml <scene.yaml> <input.bin> <output.bin>
//   force_solver_host --print-config <scene.yaml>
//
// With --solver-yaml the solver is configured from the scene file's
// `simulation.solver` node the way the reference does it
// (PrimalDualForceSolver::fillFromYAML, PrimalDualForceSolver.cpp:650-673, then
// NonSmoothContactForce / OnlyNormalForce::fillFromYAML,
// NonSmoothContactForce.cpp:320-334, OnlyNormalForce.cpp:218-230), including
// its errors; --print-config prints the resulting settings and exits (no
// device needed).  The scene file is read by a YAML subset reader (block
// mappings of scalars, `#` comments, quoted strings): the part of YAML the
// solver node uses.
//
// input.bin: int32 nb, nc; per body: pos[3] quat[4 xyzw] vel[3] ang[3] mass
// I0[3] (float64) static (uint8); per contact: objId[2] (int32) pos[3]
// frame[9] depth (float64).  output.bin: int32 status, newton_iters; per body
// dv[3] dw[3]; per contact localForce[3] (float64).
#include <cctype>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <map>
#include <memory>
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

// A node of a YAML block mapping: scalar values and child mappings by key.
struct YamlNode {
    std::map<std::string, std::string> scalars;
    std::map<std::string, std::shared_ptr<YamlNode>> maps;
    bool has(const std::string& k) const { return scalars.count(k) || maps.count(k); }
    const YamlNode* child(const std::string& k) const {
        auto it = maps.find(k);
        return it == maps.end() ? nullptr : it->second.get();
    }
};

static std::string trim(const std::string& x) {
    size_t a = 0, b = x.size();
    while (a < b && std::isspace((unsigned char)x[a])) ++a;
    while (b > a && std::isspace((unsigned char)x[b - 1])) --b;
    return x.substr(a, b - a);
}

// Block mappings only: "key: value" and "key:" opening a deeper-indented
// mapping; sequence items and flow collections are kept as raw scalars.
static YamlNode parse_yaml(const std::string& path) {
    std::ifstream in(path);
    if (!in) throw std::runtime_error("cannot open " + path);
    YamlNode root;
    std::vector<std::pair<int, YamlNode*>> stack{{-1, &root}};
    std::string line;
    while (std::getline(in, line)) {
        bool quoted = false;
        char q = 0;
        for (size_t i = 0; i < line.size(); ++i) {  // strip a comment outside quotes
            const char c = line[i];
            if (quoted) { if (c == q) quoted = false; continue; }
            if (c == '"' || c == '\'') { quoted = true; q = c; continue; }
            if (c == '#' && (i == 0 || std::isspace((unsigned char)line[i - 1]))) { line.resize(i); break; }
        }
        if (trim(line).empty()) continue;
        int indent = 0;
        while (indent < (int)line.size() && line[indent] == ' ') ++indent;
        const std::string body = trim(line);
        if (body[0] == '-') continue;  // sequence item: not used by the solver node
        const size_t colon = body.find(':');
        if (colon == std::string::npos) continue;
        const std::string key = trim(body.substr(0, colon));
        std::string val = trim(body.substr(colon + 1));
        while (stack.size() > 1 && stack.back().first >= indent) stack.pop_back();
        YamlNode* parent = stack.back().second;
        if (val.empty()) {
            auto node = std::make_shared<YamlNode>();
            parent->maps[key] = node;
            stack.push_back({indent, node.get()});
        } else {
            if (val.size() >= 2 && (val.front() == '"' || val.front() == '\'') && val.back() == val.front())
                val = val.substr(1, val.size() - 2);
            parent->scalars[key] = val;
        }
    }
    return root;
}

// parseScalar with a default (src/Common/InputParse.h:30-40): the value when
// the key holds a scalar, else the default.
static double scalar_or(const YamlNode& n, const char* k, double def) {
    auto it = n.scalars.find(k);
    if (it == n.scalars.end()) return def;
    char* end = nullptr;
    const double v = std::strtod(it->second.c_str(), &end);
    if (end == it->second.c_str()) throw std::runtime_error(std::string("bad number for '") + k + "'");
    return v;
}
static bool bool_or(const YamlNode& n, const char* k, bool def) {
    auto it = n.scalars.find(k);
    if (it == n.scalars.end()) return def;
    std::string v;
    for (char c : it->second) v += (char)std::tolower((unsigned char)c);
    if (v == "true" || v == "yes" || v == "on" || v == "y") return true;
    if (v == "false" || v == "no" || v == "off" || v == "n") return false;
    throw std::runtime_error(std::string("bad boolean for '") + k + "'");
}

class PrimalDualGpuForceSolver {
   public:
    PrimalDualGpuForceSolver(int iterations, double tolerance) {
        pdc_config_default(&cfg_);
        cfg_.max_iter = iterations;
        cfg_.tol = tolerance;
    }
    // PrimalDualForceSolver::fillFromYAML (PrimalDualForceSolver.cpp:650-673) and
    // the force model's own fillFromYAML (NonSmoothContactForce.cpp:320-334,
    // OnlyNormalForce.cpp:218-230), on the scene file's simulation.solver node.
    explicit PrimalDualGpuForceSolver(const YamlNode& node) {
        pdc_config_default(&cfg_);
        cfg_.tol = scalar_or(node, "tolerance", 1e-6);
        cfg_.max_iter = (int)scalar_or(node, "iterations", 100);
        const YamlNode* f = node.child("non_smooth_force");
        if (!f && !node.has("non_smooth_force")) throw std::runtime_error("No non-smooth force defined!");
        static const YamlNode empty;
        if (!f) f = &empty;
        auto name = f->scalars.find("name");
        if (name == f->scalars.end()) throw std::runtime_error("Non-smooth force: no name provided!");
        double def_restitution = 0.0;
        if (name->second == "non_smooth_contact") {
            cfg_.force_model = PDC_FORCE_NON_SMOOTH_CONTACT;
        } else if (name->second == "only_normal") {
            cfg_.force_model = PDC_FORCE_ONLY_NORMAL;
            def_restitution = 0.5;
        } else {  // the reference leaves its force unset here and then dereferences it
            throw std::runtime_error("Unknown non-smooth force: " + name->second);
        }
        cfg_.spring_based = bool_or(*f, "spring_based_force", false) ? 1 : 0;
        if (cfg_.spring_based) {
            cfg_.spring_k = scalar_or(*f, "spring_k", 1e6);
            cfg_.spring_damp = scalar_or(*f, "spring_damp", 0.01);
        } else {
            cfg_.restitution = scalar_or(*f, "restitution", def_restitution);
        }
        if (cfg_.force_model == PDC_FORCE_NON_SMOOTH_CONTACT) cfg_.mu = scalar_or(*f, "static_coeff", 0.5);
    }
    ~PrimalDualGpuForceSolver() { pdc_destroy(solver_); }
    const pdc_config& config() const { return cfg_; }
    void create() {
        if (pdc_create(&cfg_, &solver_) != PDC_OK) throw std::runtime_error(pdc_last_error(nullptr));
    }

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
        if (!solver_) create();
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

// The simulation.solver node of a scene file (DynamicSystem::fillFromYAML,
// DynamicSystem.cpp:385-399: the solver must be named primal_dual).
static const YamlNode& solver_node(const YamlNode& root) {
    const YamlNode* sim = root.child("simulation");
    const YamlNode* solver = sim ? sim->child("solver") : nullptr;
    if (!solver) throw std::runtime_error("No force solver specified!");
    auto name = solver->scalars.find("name");
    const std::string n = name == solver->scalars.end() ? "" : name->second;
    if (n != "primal_dual") throw std::runtime_error("No solver of name: " + n + "found!");
    return *solver;
}

int main(int argc, char** argv) {
    if (argc < 3) {
        std::fprintf(stderr,
                     "usage: %s <input.bin> <output.bin> [iterations] [tolerance]\n"
                     "       %s --solver-yaml <scene.yaml> <input.bin> <output.bin>\n"
                     "       %s --print-config <scene.yaml>\n",
                     argv[0], argv[0], argv[0]);
        return 2;
    }
    try {
        std::unique_ptr<PrimalDualGpuForceSolver> solver;
        const std::string mode = argv[1];
        if (mode == "--print-config" || mode == "--solver-yaml") {
            const YamlNode root = parse_yaml(argv[2]);
            solver = std::make_unique<PrimalDualGpuForceSolver>(solver_node(root));
            if (mode == "--print-config") {
                const pdc_config& c = solver->config();
                std::printf("tol %.17g\nmax_iter %d\nforce_model %d\nspring_based %d\nmu %.17g\n"
                            "restitution %.17g\nspring_k %.17g\nspring_damp %.17g\n",
                            c.tol, c.max_iter, c.force_model, c.spring_based, c.mu, c.restitution, c.spring_k,
                            c.spring_damp);
                return 0;
            }
            if (argc < 5) throw std::runtime_error("--solver-yaml needs <scene.yaml> <input.bin> <output.bin>");
            argv += 2;
            argc -= 2;
        }
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
        if (!solver)
            solver = std::make_unique<PrimalDualGpuForceSolver>(argc > 3 ? std::atoi(argv[3]) : 100,
                                                                argc > 4 ? std::atof(argv[4]) : 1e-6);
        const pdc_stats st = solver->fillForces(dt, g, contacts, objects);
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
