// A recorded computation over device tensors with forward (JVP) and reverse (VJP) derivative
// passes.  The CCSD residual is written once against this interface: the plain residual runs
// the recorded ops eagerly; the Jacobian transformation replays them with tangents (one extra
// trailing index over the trial vectors), the transpose transformation and the adjoints into the
// Cholesky vectors and h run them backwards.
#pragma once

#include <functional>
#include <string>
#include <vector>

#include "common.cuh"

namespace ccsd {

struct GNode {
    std::string name;
    std::vector<int64_t> dims;   // column-major, contiguous
    int64_t size = 1;
    double *v = nullptr;         // primal value
    DBuf own;                    // storage when the graph owns the primal
    DBuf tan, adj;               // [size x nvec]
    bool active = false;         // depends on a differentiated input
    bool zero = false;           // allocated by zeros() and not written yet: reads as zero, and the
                                 // first op writing it overwrites instead of accumulating
    int last_use = -1;           // index of the last op reading this node
};

enum class OpKind { Contract, Permute, Squareup, PackHalf, PackSym, Trace, Custom };

// A custom op supplies its own forward / tangent / adjoint callbacks.
struct CustomOp {
    std::function<void()> forward;
    std::function<void(int nvec)> tangent;   // reads input tangents, accumulates out tangent
    std::function<void(int nvec)> adjoint;   // reads out adjoint, accumulates input adjoints
};

struct GOp {
    OpKind kind;
    int out = -1, a = -1, b = -1;
    double alpha = 1.0;
    std::string spec;            // contract: "la,lb->lc"; permute: "lin->lout"
    bool fp64 = false;           // force FP64 (first-order terms)
    int custom = -1;
};

// packed[(M, m)] += (full[M, m] + full[m, M]) * (1/2 if M == m) over M >= m: the symmetrised full
// doubles array packed as eT's symmetric_sum + scale_diagonal(1/2) + packin do, in one pass
void pack_sym_add(Exec &ex, const double *full, double *packed, int64_t nov);

class Graph {
  public:
    explicit Graph(Exec &ex) : ex_(ex) {}
    Graph(const Graph &) = delete;
    Graph &operator=(const Graph &) = delete;

    // node creation
    int input(const std::string &name, std::vector<int64_t> dims, const double *p);
    int zeros(const std::string &name, std::vector<int64_t> dims);
    int alias(int node);   // same value (e.g. an unchanged block)

    // out += alpha * einsum(spec, a, b)
    void contract(int out, const char *spec, double alpha, int a, int b, bool fp64 = false);
    // out += alpha * permute(a), spec "ajbi->aibj" (labels name the dims of a / out)
    void permute(int out, const char *spec, double alpha, int a);
    // out(full (v,o,v,o) symmetric) += squareup(a packed)
    void squareup(int out, int a);
    // out(packed) += pack with the diagonal halved of a (full; read triangle (m, M))
    void pack_half(int out, int a);
    // out(packed) += pack with the diagonal halved of a + a^T (a full, not symmetric): eT's
    // symmetric_sum, scale_diagonal(1/2) and packin in one pass
    void pack_sym(int out, int a);
    // out[J] += sum_k a[J, k, k]
    void trace(int out, int a);
    // custom op over existing nodes
    int custom(CustomOp op, int out, std::vector<int> ins);

    GNode &node(int i) {
        materialize(i);
        return nodes_[i];
    }
    const double *value(int i) {
        materialize(i);
        return nodes_[i].v;
    }
    int64_t nov = 0;               // for squareup / pack_half

    // derivative passes; seeds are [size x nvec] device arrays for the listed nodes.  Each pass
    // starts from zero tangents / adjoints, so a recording can serve several passes.
    void mark_active(const std::vector<int> &inputs);
    void clear_derivatives();
    void jvp(const std::vector<int> &inputs, const std::vector<const double *> &seeds, int nvec,
             const std::vector<int> &outputs, const std::vector<double *> &results);
    void vjp(const std::vector<int> &outputs, const std::vector<const double *> &seeds, int nvec,
             const std::vector<int> &inputs, const std::vector<double *> &results);

    // helpers for custom ops
    double *tangent(int i, int nvec);   // allocates (zeroed) on first use
    double *adjoint(int i, int nvec);
    bool has_tangent(int i) const { return (bool)nodes_[i].tan; }
    bool has_adjoint(int i) const { return (bool)nodes_[i].adj; }
    Exec &exec() { return ex_; }

  private:
    Exec &ex_;
    std::vector<GNode> nodes_;
    std::vector<GOp> ops_;
    std::vector<CustomOp> customs_;
    std::vector<std::vector<int>> custom_ins_;
    void run_forward(const GOp &op);
    TV view(int node) const;
    // fills a node that zeros() allocated and nothing has written yet
    void materialize(int node);
    TV tview(int node, int nvec, bool adjoint);
};

}  // namespace ccsd
