// adjoint_gen.cpp -- build step: writes csrc/adjoint_ops.gen.cuh, the
// reverse-mode (adjoint) code of the per-node K17 collision operator.
//
// The K17 operator of csrc/collision_math.cuh is a template over the
// arithmetic type.  This program instantiates it with a recording type
// (Sym) on the host: every arithmetic operation the operator performs appends
// one node to a tape, so the tape is exactly the operation sequence the
// forward kernels run (FP64 and FP32 forms are traced separately; they differ
// in constants and in the FP32-only rearrangements of the operator).  From
// the tape it emits, per precision, a device function
//
//   k17Adjoint(a[27], lam[27], rates, fx, fy, fz, gfx, gfy, gfz)
//
// that recomputes the forward values from the pre-collision populations a[]
// and then applies the transposed Jacobian: on entry lam[d] is the adjoint of
// the post-collision population of direction d, on return the adjoint of the
// pre-collision population of direction d; g{x,y,z} receive the adjoint of
// the half-force inputs.  The reverse sweep is the textbook one (each
// operation's partial derivatives, accumulated in reverse tape order); |x|
// has derivative sign(x).  Values of nodes that do not reach an output are
// never emitted.
//
// Build: g++ -std=c++17 -I<cuda>/include adjoint_gen.cpp -o adjoint_gen (host code
// only; the operator header's __host__ __device__ marks are empty there), run
// as ./adjoint_gen <output header>.  virtualfluids_b200/build.py does this
// when the generator or collision_math.cuh is newer than the header.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <map>
#include <string>
#include <vector>

namespace vfgen
{
enum Op { INPUT, PARAM, CONST, ADD, SUB, MUL, DIV, FDIV, NEG, FMA, ABS };

struct Node {
    Op op;
    int a = -1, b = -1, c = -1;
    double k = 0.0;   // CONST value (already rounded to the traced precision)
    std::string name; // INPUT / PARAM expression
};

struct Tape {
    std::vector<Node> nodes;
    bool single = false; // constants and folding in float
    int push(const Node& n)
    {
        nodes.push_back(n);
        return (int)nodes.size() - 1;
    }
};
static Tape* tape = nullptr;

double roundTo(double v) { return tape->single ? (double)(float)v : v; }

struct Sym {
    int id;
    Sym() : id(-1) {}
    explicit Sym(int i, bool) : id(i) {}
    Sym(double v)
    {
        Node n;
        n.op = CONST;
        n.k = roundTo(v);
        id = tape->push(n);
    }
    Sym(float v) : Sym((double)v) {}
    Sym(int v) : Sym((double)v) {}
};

inline bool isConst(const Sym& s) { return tape->nodes[s.id].op == CONST; }
inline double cval(const Sym& s) { return tape->nodes[s.id].k; }

inline Sym make(Op op, const Sym& a, const Sym& b = Sym(), const Sym& c = Sym())
{
    // fold operations on constants in the traced precision
    const bool ca = isConst(a), cb = b.id < 0 || isConst(b), cc = c.id < 0 || isConst(c);
    if (ca && cb && cc) {
        const double x = cval(a), y = b.id >= 0 ? cval(b) : 0.0, z = c.id >= 0 ? cval(c) : 0.0;
        double r = 0.0;
        if (tape->single) {
            const float fx = (float)x, fy = (float)y, fz = (float)z;
            switch (op) {
            case ADD: r = fx + fy; break;
            case SUB: r = fx - fy; break;
            case MUL: r = fx * fy; break;
            case DIV:
            case FDIV: r = fx / fy; break;
            case NEG: r = -fx; break;
            case FMA: r = std::fmaf(fx, fy, fz); break;
            case ABS: r = std::fabs(fx); break;
            default: std::abort();
            }
        } else {
            switch (op) {
            case ADD: r = x + y; break;
            case SUB: r = x - y; break;
            case MUL: r = x * y; break;
            case DIV:
            case FDIV: r = x / y; break;
            case NEG: r = -x; break;
            case FMA: r = std::fma(x, y, z); break;
            case ABS: r = std::fabs(x); break;
            default: std::abort();
            }
        }
        return Sym(r);
    }
    Node n;
    n.op = op;
    n.a = a.id;
    n.b = b.id;
    n.c = c.id;
    return Sym(tape->push(n), true);
}

inline Sym operator+(const Sym& a, const Sym& b) { return make(ADD, a, b); }
inline Sym operator-(const Sym& a, const Sym& b) { return make(SUB, a, b); }
inline Sym operator*(const Sym& a, const Sym& b) { return make(MUL, a, b); }
inline Sym operator/(const Sym& a, const Sym& b) { return make(DIV, a, b); }
inline Sym operator-(const Sym& a) { return make(NEG, a); }
inline Sym& operator+=(Sym& a, const Sym& b) { return a = a + b; }
inline Sym& operator-=(Sym& a, const Sym& b) { return a = a - b; }
inline Sym& operator*=(Sym& a, const Sym& b) { return a = a * b; }
inline Sym fma(const Sym& a, const Sym& b, const Sym& c) { return make(FMA, a, b, c); }
inline Sym fabs(const Sym& a) { return make(ABS, a); }

Sym input(const std::string& name, Op op = INPUT)
{
    Node n;
    n.op = op;
    n.name = name;
    return Sym(tape->push(n), true);
}
} // namespace vfgen

// the operator source, instantiated below with the recording type
#include "../csrc/collision_math.cuh"

namespace vfb
{
template <>
struct ScalarOf<vfgen::Sym> {
    using type = double;
};
// the FP32 trace: constants are float (cst<R> and the chimera K values)
struct SymF : vfgen::Sym {
    using Sym::Sym;
    SymF(const vfgen::Sym& s) : Sym(s) {}
};
template <>
__host__ __device__ inline vfgen::Sym limiterQuotient<vfgen::Sym>(vfgen::Sym x, vfgen::Sym y)
{
    return vfgen::make(vfgen::FDIV, x, y);
}
} // namespace vfb

namespace vfgen
{
struct Emitter {
    const Tape& t;
    std::string real;          // "float" / "double"
    std::vector<int> outputs;  // tape ids of the 27 post-collision values
    std::vector<int> forceIds; // tape ids of fx, fy, fz
    std::vector<int> inputIds; // tape ids of a[0..26]
    std::vector<bool> live;

    std::string lit(double v) const
    {
        char buf[64];
        if (real == "float")
            std::snprintf(buf, sizeof buf, "%.9gf", v);
        else
            std::snprintf(buf, sizeof buf, "%.17g", v);
        std::string s(buf);
        if (s.find_first_of(".eEn") == std::string::npos) // integral value: keep it a floating literal
            s.insert(real == "float" ? s.size() - 1 : s.size(), ".0");
        return "R(" + s + ")";
    }
    std::string val(int id) const
    {
        const Node& n = t.nodes[id];
        if (n.op == CONST)
            return lit(n.k);
        if (n.op == INPUT || n.op == PARAM)
            return n.name;
        return "v" + std::to_string(id);
    }

    void markLive()
    {
        live.assign(t.nodes.size(), false);
        std::vector<int> stack(outputs.begin(), outputs.end());
        while (!stack.empty()) {
            const int i = stack.back();
            stack.pop_back();
            if (i < 0 || live[i])
                continue;
            live[i] = true;
            const Node& n = t.nodes[i];
            for (int o : { n.a, n.b, n.c })
                if (o >= 0)
                    stack.push_back(o);
        }
    }

    std::string forwardExpr(const Node& n) const
    {
        switch (n.op) {
        case ADD: return val(n.a) + " + " + val(n.b);
        case SUB: return val(n.a) + " - " + val(n.b);
        case MUL: return val(n.a) + " * " + val(n.b);
        case DIV: return val(n.a) + " / " + val(n.b);
        case FDIV: return "limiterQuotient<R>(" + val(n.a) + ", " + val(n.b) + ")";
        case NEG: return "-" + val(n.a);
        case FMA: return "fma(" + val(n.a) + ", " + val(n.b) + ", " + val(n.c) + ")";
        case ABS: return "fabs(" + val(n.a) + ")";
        default: std::abort();
        }
    }

    // adjoint accumulation targets: inputs, the force parameters and computed nodes
    bool wantsAdjoint(int id) const
    {
        const Node& n = t.nodes[id];
        if (n.op == CONST)
            return false;
        if (n.op == PARAM) {
            for (int f : forceIds)
                if (f == id)
                    return true;
            return false;
        }
        return true;
    }

    void emit(FILE* out, const char* fname)
    {
        markLive();
        const char* rs = real.c_str();
        std::fprintf(out,
                         "template <>\n__host__ __device__ __forceinline__ void %s<%s>(const %s* __restrict__ a, "
                         "%s* lam,\n    const K17Rates<%s>& r, %s fx, %s fy, %s fz, %s& gfx, %s& gfy, %s& gfz)\n{\n",
                         fname, rs, rs, rs, rs, rs, rs, rs, rs, rs, rs);
        std::fprintf(out, "    using R = %s;\n", real.c_str());
        int nf = 0, nr = 0;
        for (size_t i = 0; i < t.nodes.size(); ++i) {
            const Node& n = t.nodes[i];
            if (!live[i] || n.op == INPUT || n.op == PARAM || n.op == CONST)
                continue;
            std::fprintf(out, "    const R v%zu = %s;\n", i, forwardExpr(n).c_str());
            ++nf;
        }
        // reverse sweep
        std::map<int, bool> started; // adjoint variable declared
        auto acc = [&](int id, const std::string& expr, bool negate) {
            if (id < 0 || !wantsAdjoint(id))
                return;
            const std::string g = "g" + std::to_string(id);
            if (!started[id]) {
                std::fprintf(out, "    R %s = %s%s;\n", g.c_str(), negate ? "-" : "", expr.c_str());
                started[id] = true;
            } else {
                std::fprintf(out, "    %s %s= %s;\n", g.c_str(), negate ? "-" : "+", expr.c_str());
            }
            ++nr;
        };
        // seeds: lam[d] is the adjoint of output d (an output node may appear once)
        for (int d = 0; d < 27; ++d)
            acc(outputs[d], "lam[" + std::to_string(d) + "]", false);
        for (int i = (int)t.nodes.size() - 1; i >= 0; --i) {
            const Node& n = t.nodes[i];
            if (!live[i] || !started[i] || n.op == INPUT || n.op == PARAM || n.op == CONST)
                continue;
            const std::string g = "g" + std::to_string(i);
            switch (n.op) {
            case ADD:
                acc(n.a, g, false);
                acc(n.b, g, false);
                break;
            case SUB:
                acc(n.a, g, false);
                acc(n.b, g, true);
                break;
            case MUL:
                acc(n.a, g + " * " + val(n.b), false);
                acc(n.b, g + " * " + val(n.a), false);
                break;
            case DIV:
            case FDIV: {
                // q = a / b: dq/da = 1/b, dq/db = -q/b
                const std::string s = "s" + std::to_string(i);
                std::fprintf(out, "    const R %s = %s / %s;\n", s.c_str(), g.c_str(), val(n.b).c_str());
                acc(n.a, s, false);
                acc(n.b, s + " * " + val(i), true);
                break;
            }
            case NEG: acc(n.a, g, true); break;
            case FMA:
                acc(n.a, g + " * " + val(n.b), false);
                acc(n.b, g + " * " + val(n.a), false);
                acc(n.c, g, false);
                break;
            case ABS:
                acc(n.a, "(" + val(n.a) + " > R(0) ? " + g + " : " + val(n.a) + " < R(0) ? -" + g + " : R(0))",
                    false);
                break;
            default: std::abort();
            }
        }
        for (int d = 0; d < 27; ++d)
            std::fprintf(out, "    lam[%d] = %s;\n", d,
                         started[inputIds[d]] ? ("g" + std::to_string(inputIds[d])).c_str() : "R(0)");
        const char* gn[3] = { "gfx", "gfy", "gfz" };
        for (int c = 0; c < 3; ++c)
            std::fprintf(out, "    %s = %s;\n", gn[c],
                         forceIds.size() > (size_t)c && started[forceIds[c]]
                             ? ("g" + std::to_string(forceIds[c])).c_str()
                             : "R(0)");
        std::fprintf(out, "}\n// %d forward and %d reverse operations\n\n", nf, nr);
        std::fprintf(stderr, "%s<%s>: %d forward, %d reverse operations\n", fname, real.c_str(), nf, nr);
    }
};

template <class R>
void traceK17(Tape& tp, bool single, Emitter& em)
{
    tape = &tp;
    tp.single = single;
    R f[27];
    for (int d = 0; d < 27; ++d) {
        f[d] = input("a[" + std::to_string(d) + "]");
        em.inputIds.push_back(f[d].id);
    }
    vfb::K17Rates<R> r;
    const char* names[] = { "r.omega", "r.OxyyPxzz", "r.OxyyMxzz", "r.Oxyz", "r.oneMinusOxyyPxzz",
                            "r.oneMinusOxyyMxzz", "r.oneMinusOxyz", "r.factorA", "r.factorB", "r.minusTau",
                            "r.halfMinusOmega", "r.omegaThreeHalves", "r.minusThreeOmega",
                            "r.secondOrderCorrection", "r.qlP", "r.qlM", "r.qlD", "r.fourthA", "r.fourthB" };
    R* fields[] = { &r.omega, &r.OxyyPxzz, &r.OxyyMxzz, &r.Oxyz, &r.oneMinusOxyyPxzz, &r.oneMinusOxyyMxzz,
                    &r.oneMinusOxyz, &r.factorA, &r.factorB, &r.minusTau, &r.halfMinusOmega, &r.omegaThreeHalves,
                    &r.minusThreeOmega, &r.secondOrderCorrection, &r.qlP, &r.qlM, &r.qlD, &r.fourthA, &r.fourthB };
    for (size_t i = 0; i < sizeof(fields) / sizeof(fields[0]); ++i)
        *fields[i] = input(names[i], PARAM);
    R fx = input("fx", PARAM), fy = input("fy", PARAM), fz = input("fz", PARAM);
    em.forceIds = { fx.id, fy.id, fz.id };
    R drho, vx, vy, vz;
    vfb::k17Collide(f, r, fx, fy, fz, drho, vx, vy, vz);
    for (int d = 0; d < 27; ++d)
        em.outputs.push_back(f[d].id);
}

} // namespace vfgen

// the FP32 trace needs float constants: ScalarOf<SymF> = float
namespace vfb
{
template <>
struct ScalarOf<SymF> {
    using type = float;
};
} // namespace vfb

namespace vfb
{
inline SymF operator+(const SymF& a, const SymF& b) { return vfgen::make(vfgen::ADD, a, b); }
inline SymF operator-(const SymF& a, const SymF& b) { return vfgen::make(vfgen::SUB, a, b); }
inline SymF operator*(const SymF& a, const SymF& b) { return vfgen::make(vfgen::MUL, a, b); }
inline SymF operator/(const SymF& a, const SymF& b) { return vfgen::make(vfgen::DIV, a, b); }
inline SymF operator-(const SymF& a) { return vfgen::make(vfgen::NEG, a); }
inline SymF& operator+=(SymF& a, const SymF& b) { return a = a + b; }
inline SymF& operator-=(SymF& a, const SymF& b) { return a = a - b; }
inline SymF fma(const SymF& a, const SymF& b, const SymF& c) { return vfgen::make(vfgen::FMA, a, b, c); }
inline SymF fabs(const SymF& a) { return vfgen::make(vfgen::ABS, a); }
template <>
__host__ __device__ inline SymF limiterQuotient<SymF>(SymF x, SymF y)
{
    return vfgen::make(vfgen::FDIV, x, y);
}
} // namespace vfb

int main(int argc, char** argv)
{
    if (argc != 2) {
        std::fprintf(stderr, "usage: %s <output header>\n", argv[0]);
        return 2;
    }
    FILE* out = std::fopen(argv[1], "w");
    if (!out)
        return 1;
    std::fprintf(out,
                 "// adjoint_ops.gen.cuh -- GENERATED by virtualfluids_b200/gen/adjoint_gen.cpp from the K17\n"
                 "// operator of collision_math.cuh; do not edit.  The forward recomputation and\n"
                 "// the reverse sweep of one node's collision, per precision.\n"
                 "#pragma once\n\n#include \"collision_math.cuh\"\n\nnamespace vfb\n{\n"
                 "template <class R>\n__host__ __device__ void k17Adjoint(const R* __restrict__ a, R* lam, "
                 "const K17Rates<R>& r, R fx, R fy, R fz, R& gfx, R& gfy, R& gfz);\n"
                 "\n");
    {
        vfgen::Tape tp;
        vfgen::Emitter em{ tp, "double" };
        vfgen::traceK17<vfgen::Sym>(tp, false, em);
        em.emit(out, "k17Adjoint");
    }
    {
        vfgen::Tape tp;
        vfgen::Emitter em{ tp, "float" };
        vfgen::traceK17<vfb::SymF>(tp, true, em);
        em.emit(out, "k17Adjoint");
    }
    std::fprintf(out, "} // namespace vfb\n");
    std::fclose(out);
    return 0;
}
