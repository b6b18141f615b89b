// Recorded tensor computation with forward- and reverse-mode derivative passes.
#include <algorithm>

#include "graph.cuh"
#include "tensor_ops.cuh"

namespace ccsd {

namespace {

constexpr char BATCH = '#';   // label of the trailing trial index of tangents / adjoints

#define GRID_STRIDE(i, total) \
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < (total); i += (int64_t)gridDim.x * blockDim.x)

inline int grid_for(int64_t total, int block) {
    int64_t g = (total + block - 1) / block;
    return (int)std::max<int64_t>(1, std::min<int64_t>(g, 148 * 64));
}

__device__ __forceinline__ void untri(int64_t idx, int64_t &M, int64_t &m) {
    int64_t r = (int64_t)((sqrt(8.0 * (double)idx + 1.0) - 1.0) * 0.5);
    while (r * (r + 1) / 2 > idx) r--;
    while ((r + 1) * (r + 2) / 2 <= idx) r++;
    M = r;
    m = idx - r * (r + 1) / 2;
}

// packed += S^T full over nbatch columns: p[(M,m)] += F[M,m] + F[m,M] (M > m), F[M,M] (M == m)
__global__ void squareup_adj_kernel(const double *__restrict__ full, double *__restrict__ packed, int64_t nov,
                                    int64_t nbatch) {
    const int64_t np = nov * (nov + 1) / 2;
    GRID_STRIDE(idx, np * nbatch) {
        int64_t n = idx / np, p = idx - n * np, M, m;
        untri(p, M, m);
        const double *F = full + n * nov * nov;
        double v = F[M + nov * m];
        if (M != m) v += F[m + nov * M];
        packed[idx] += v;
    }
}

// full(m, M) += p[(M, m)] * (1/2 if M == m)  (adjoint of the packing read of pack_half_diag_add)
__global__ void pack_half_adj_kernel(const double *__restrict__ packed, double *__restrict__ full, int64_t nov,
                                     int64_t nbatch) {
    const int64_t np = nov * (nov + 1) / 2;
    GRID_STRIDE(idx, np * nbatch) {
        int64_t n = idx / np, p = idx - n * np, M, m;
        untri(p, M, m);
        double v = packed[idx];
        if (M == m) v *= 0.5;
        full[n * nov * nov + m + nov * M] += v;
    }
}

__global__ void pack_half_batch_kernel(const double *__restrict__ full, double *__restrict__ packed, int64_t nov,
                                       int64_t nbatch) {
    const int64_t np = nov * (nov + 1) / 2;
    GRID_STRIDE(idx, np * nbatch) {
        int64_t n = idx / np, p = idx - n * np, M, m;
        untri(p, M, m);
        double v = full[n * nov * nov + m + nov * M];
        if (M == m) v *= 0.5;
        packed[idx] += v;
    }
}

// packed[(M, m)] += (F[m, M] + F[M, m]) * (1/2 if M == m): consecutive threads take consecutive m
// of one M, so the F[m, M] reads are coalesced and the F[M, m] reads of neighbouring M share sectors
// in L2
__global__ void pack_sym_batch_kernel(const double *__restrict__ full, double *__restrict__ packed, int64_t nov,
                                      int64_t nbatch) {
    const int64_t np = nov * (nov + 1) / 2;
    GRID_STRIDE(idx, np * nbatch) {
        int64_t n = idx / np, p = idx - n * np, M, m;
        untri(p, M, m);
        const double *F = full + n * nov * nov;
        const double v = F[m + nov * M] + F[M + nov * m];
        packed[idx] += M == m ? 0.5 * v : v;
    }
}

// full (+)= the symmetric square of packed (accumulate = 0: overwrite)
__global__ void squareup_batch_kernel(const double *__restrict__ packed, double *__restrict__ full, int64_t nov,
                                      int64_t nbatch, int accumulate) {
    const int64_t nf = nov * nov, np = nov * (nov + 1) / 2;
    GRID_STRIDE(idx, nf * nbatch) {
        int64_t n = idx / nf, r = idx - n * nf;
        int64_t x = r % nov, y = r / nov;
        int64_t M = x > y ? x : y, m = x > y ? y : x;
        const double v = packed[n * np + M * (M + 1) / 2 + m];
        full[idx] = accumulate ? full[idx] + v : v;
    }
}

// out[J, n] += sum_k a[J, k, k, n]  /  adjoint: a[J, k, k, n] += out[J, n]
__global__ void trace_batch_kernel(const double *__restrict__ a, double *__restrict__ out, int64_t nJ, int64_t no,
                                   int64_t nbatch, int adjoint) {
    GRID_STRIDE(idx, nJ * nbatch) {
        int64_t J = idx % nJ, n = idx / nJ;
        if (!adjoint) {
            double s = 0.0;
            for (int64_t k = 0; k < no; k++) s += a[n * nJ * no * no + J + nJ * (k + no * k)];
            out[idx] += s;
        } else {
            double v = a[idx];   // here a is the adjoint of out (nJ x nbatch)
            for (int64_t k = 0; k < no; k++) out[n * nJ * no * no + J + nJ * (k + no * k)] += v;
        }
    }
}

std::string with_batch(const std::string &labels) { return labels + BATCH; }

// An op recorded as FP64 (the first-order terms of the mixed residual) runs in FP64 arithmetic; in a
// mixed-precision evaluation its large products go to the int8 digit GEMM (ex.mixed_fp64_digits
// digits, FP64-accurate) rather than DGEMM, unless the caller already chose the FP64 arithmetic.
struct Fp64Scope {
    Exec &ex;
    Prec prec;
    int digits;
    Fp64Scope(Exec &e, bool on) : ex(e), prec(e.prec), digits(e.fp64_digits) {
        if (!on) return;
        if (prec == Prec::MIXED && ex.fp64_digits == 0) ex.fp64_digits = ex.mixed_fp64_digits;
        ex.prec = Prec::FP64;
    }
    ~Fp64Scope() {
        ex.prec = prec;
        ex.fp64_digits = digits;
    }
    Fp64Scope(const Fp64Scope &) = delete;
    Fp64Scope &operator=(const Fp64Scope &) = delete;
};

}  // namespace

int Graph::input(const std::string &name, std::vector<int64_t> dims, const double *p) {
    GNode n;
    n.name = name;
    n.dims = std::move(dims);
    for (int64_t d : n.dims) n.size *= d;
    n.v = const_cast<double *>(p);
    nodes_.push_back(std::move(n));
    return (int)nodes_.size() - 1;
}

int Graph::zeros(const std::string &name, std::vector<int64_t> dims) {
    GNode n;
    n.name = name;
    n.dims = std::move(dims);
    for (int64_t d : n.dims) n.size *= d;
    n.own = dalloc(n.size, ex_.stream);
    n.v = n.own.d();
    n.zero = true;
    nodes_.push_back(std::move(n));
    return (int)nodes_.size() - 1;
}

void Graph::materialize(int i) {
    GNode &n = nodes_[i];
    if (!n.zero) return;
    fill(ex_, n.v, n.size, 0.0);
    n.zero = false;
}

int Graph::alias(int node) { return node; }

TV Graph::view(int i) const {
    const GNode &n = nodes_[i];
    TV v;
    v.p = n.v;
    v.nd = (int)n.dims.size();
    int64_t st = 1;
    for (int k = 0; k < v.nd; k++) {
        v.n[k] = n.dims[k];
        v.s[k] = st;
        st *= n.dims[k];
    }
    return v;
}

TV Graph::tview(int i, int nvec, bool adj) {
    TV v = view(i);
    v.p = adj ? adjoint(i, nvec) : tangent(i, nvec);
    v.n[v.nd] = nvec;
    v.s[v.nd] = nodes_[i].size;
    v.nd++;
    return v;
}

double *Graph::tangent(int i, int nvec) {
    GNode &n = nodes_[i];
    if (!n.tan) {
        n.tan = dalloc(n.size * nvec, ex_.stream);
        fill(ex_, n.tan.d(), n.size * nvec, 0.0);
    }
    return n.tan.d();
}

double *Graph::adjoint(int i, int nvec) {
    GNode &n = nodes_[i];
    if (!n.adj) {
        n.adj = dalloc(n.size * nvec, ex_.stream);
        fill(ex_, n.adj.d(), n.size * nvec, 0.0);
    }
    return n.adj.d();
}

void Graph::run_forward(const GOp &op) {
    Fp64Scope fp64(ex_, op.fp64);
    // inputs never written read as zero; an output never written is overwritten (beta = 0) by the
    // ops that write every element of it, and zero-filled first for the others
    if (op.a >= 0) materialize(op.a);
    if (op.b >= 0) materialize(op.b);
    if (op.kind == OpKind::Custom)
        for (int i : custom_ins_[op.custom]) materialize(i);
    const bool fresh = nodes_[op.out].zero &&
                       (op.kind == OpKind::Contract || op.kind == OpKind::Permute || op.kind == OpKind::Squareup);
    if (fresh) nodes_[op.out].zero = false;
    else materialize(op.out);
    const double beta = fresh ? 0.0 : 1.0;
    switch (op.kind) {
    case OpKind::Contract:
        ccsd::contract(ex_, op.spec.c_str(), op.alpha, view(op.a), view(op.b), beta, view(op.out));
        break;
    case OpKind::Permute: {
        std::string s = op.spec;
        size_t ar = s.find("->");
        std::string lin = s.substr(0, ar), lout = s.substr(ar + 2);
        TV in = view(op.a), out = view(op.out), pin;
        pin.p = in.p;
        pin.nd = out.nd;
        for (int k = 0; k < out.nd; k++) {
            size_t pos = lin.find(lout[k]);
            REQUIRE(pos != std::string::npos, CCSD_GPU_EINVAL, "permute: bad spec " + s);
            pin.n[k] = in.n[pos];
            pin.s[k] = in.s[pos];
        }
        permute_add(ex_, op.alpha, pin, beta, out);
        break;
    }
    case OpKind::Squareup:
        squareup_batch_kernel<<<grid_for(nov * nov, 256), 256, 0, ex_.stream>>>(nodes_[op.a].v, nodes_[op.out].v, nov,
                                                                                1, fresh ? 0 : 1);
        ex_.launches++;
        break;
    case OpKind::PackHalf:
        pack_half_batch_kernel<<<grid_for(nov * (nov + 1) / 2, 256), 256, 0, ex_.stream>>>(
            nodes_[op.a].v, nodes_[op.out].v, nov, 1);
        ex_.launches++;
        break;
    case OpKind::PackSym:
        pack_sym_batch_kernel<<<grid_for(nov * (nov + 1) / 2, 256), 256, 0, ex_.stream>>>(
            nodes_[op.a].v, nodes_[op.out].v, nov, 1);
        ex_.launches++;
        break;
    case OpKind::Trace: {
        const GNode &a = nodes_[op.a];
        trace_batch_kernel<<<grid_for(a.dims[0], 128), 128, 0, ex_.stream>>>(a.v, nodes_[op.out].v, a.dims[0],
                                                                              a.dims[1], 1, 0);
        ex_.launches++;
        break;
    }
    case OpKind::Custom:
        customs_[op.custom].forward();
        break;
    }
    CU_CHECK(cudaGetLastError());
}

void Graph::contract(int out, const char *spec, double alpha, int a, int b, bool fp64) {
    GOp op;
    op.kind = OpKind::Contract;
    op.out = out;
    op.a = a;
    op.b = b;
    op.alpha = alpha;
    op.spec = spec;
    op.fp64 = fp64;
    run_forward(op);
    nodes_[a].last_use = nodes_[b].last_use = (int)ops_.size();
    ops_.push_back(op);
}

void Graph::permute(int out, const char *spec, double alpha, int a) {
    GOp op;
    op.kind = OpKind::Permute;
    op.out = out;
    op.a = a;
    op.alpha = alpha;
    op.spec = spec;
    run_forward(op);
    nodes_[a].last_use = (int)ops_.size();
    ops_.push_back(op);
}

void Graph::squareup(int out, int a) {
    GOp op;
    op.kind = OpKind::Squareup;
    op.out = out;
    op.a = a;
    run_forward(op);
    nodes_[a].last_use = (int)ops_.size();
    ops_.push_back(op);
}

void Graph::pack_sym(int out, int a) {
    GOp op;
    op.kind = OpKind::PackSym;
    op.out = out;
    op.a = a;
    run_forward(op);
    nodes_[a].last_use = (int)ops_.size();
    ops_.push_back(op);
}

void Graph::pack_half(int out, int a) {
    GOp op;
    op.kind = OpKind::PackHalf;
    op.out = out;
    op.a = a;
    run_forward(op);
    nodes_[a].last_use = (int)ops_.size();
    ops_.push_back(op);
}

void Graph::trace(int out, int a) {
    GOp op;
    op.kind = OpKind::Trace;
    op.out = out;
    op.a = a;
    run_forward(op);
    nodes_[a].last_use = (int)ops_.size();
    ops_.push_back(op);
}

int Graph::custom(CustomOp c, int out, std::vector<int> ins) {
    customs_.push_back(std::move(c));
    custom_ins_.push_back(ins);
    GOp op;
    op.kind = OpKind::Custom;
    op.out = out;
    op.custom = (int)customs_.size() - 1;
    run_forward(op);
    for (int i : ins) nodes_[i].last_use = (int)ops_.size();
    ops_.push_back(op);
    return op.custom;
}

void Graph::mark_active(const std::vector<int> &inputs) {
    for (auto &n : nodes_) n.active = false;
    for (int i : inputs) nodes_[i].active = true;
    for (const GOp &op : ops_) {
        bool act = false;
        if (op.kind == OpKind::Custom) {
            for (int i : custom_ins_[op.custom]) act = act || nodes_[i].active;
        } else {
            act = nodes_[op.a].active || (op.b >= 0 && nodes_[op.b].active);
        }
        if (act) nodes_[op.out].active = true;
    }
}

void Graph::clear_derivatives() {
    for (auto &n : nodes_) {
        n.tan.release();
        n.adj.release();
    }
}

void Graph::jvp(const std::vector<int> &inputs, const std::vector<const double *> &seeds, int nvec,
                const std::vector<int> &outputs, const std::vector<double *> &results) {
    clear_derivatives();
    mark_active(inputs);
    for (size_t k = 0; k < inputs.size(); k++) {
        double *t = tangent(inputs[k], nvec);
        CU_CHECK(cudaMemcpyAsync(t, seeds[k], sizeof(double) * nodes_[inputs[k]].size * nvec,
                                 cudaMemcpyDeviceToDevice, ex_.stream));
    }
    for (const GOp &op : ops_) {
        if (!nodes_[op.out].active) continue;
        Fp64Scope fp64(ex_, op.fp64);
        switch (op.kind) {
        case OpKind::Contract: {
            std::string s = op.spec;
            size_t comma = s.find(','), ar = s.find("->");
            std::string la = s.substr(0, comma), lb = s.substr(comma + 1, ar - comma - 1), lc = s.substr(ar + 2);
            TV out = tview(op.out, nvec, false);
            if (nodes_[op.a].active) {
                std::string sp = with_batch(la) + "," + lb + "->" + with_batch(lc);
                ccsd::contract(ex_, sp.c_str(), op.alpha, tview(op.a, nvec, false), view(op.b), 1.0, out);
            }
            if (nodes_[op.b].active) {
                std::string sp = la + "," + with_batch(lb) + "->" + with_batch(lc);
                ccsd::contract(ex_, sp.c_str(), op.alpha, view(op.a), tview(op.b, nvec, false), 1.0, out);
            }
            break;
        }
        case OpKind::Permute: {
            if (!nodes_[op.a].active) break;
            size_t ar = op.spec.find("->");
            std::string lin = op.spec.substr(0, ar) + BATCH, lout = op.spec.substr(ar + 2) + BATCH;
            TV in = tview(op.a, nvec, false), out = tview(op.out, nvec, false), pin;
            pin.p = in.p;
            pin.nd = out.nd;
            for (int k = 0; k < out.nd; k++) {
                size_t pos = lin.find(lout[k]);
                pin.n[k] = in.n[pos];
                pin.s[k] = in.s[pos];
            }
            permute_add(ex_, op.alpha, pin, 1.0, out);
            break;
        }
        case OpKind::Squareup:
            if (!nodes_[op.a].active) break;
            squareup_batch_kernel<<<grid_for(nov * nov * nvec, 256), 256, 0, ex_.stream>>>(
                tangent(op.a, nvec), tangent(op.out, nvec), nov, nvec, 1);
            ex_.launches++;
            break;
        case OpKind::PackHalf:
            if (!nodes_[op.a].active) break;
            pack_half_batch_kernel<<<grid_for(nov * (nov + 1) / 2 * nvec, 256), 256, 0, ex_.stream>>>(
                tangent(op.a, nvec), tangent(op.out, nvec), nov, nvec);
            ex_.launches++;
            break;
        case OpKind::PackSym:
            if (!nodes_[op.a].active) break;
            pack_sym_batch_kernel<<<grid_for(nov * (nov + 1) / 2 * nvec, 256), 256, 0, ex_.stream>>>(
                tangent(op.a, nvec), tangent(op.out, nvec), nov, nvec);
            ex_.launches++;
            break;
        case OpKind::Trace: {
            if (!nodes_[op.a].active) break;
            const GNode &a = nodes_[op.a];
            trace_batch_kernel<<<grid_for(a.dims[0] * nvec, 128), 128, 0, ex_.stream>>>(
                tangent(op.a, nvec), tangent(op.out, nvec), a.dims[0], a.dims[1], nvec, 0);
            ex_.launches++;
            break;
        }
        case OpKind::Custom:
            customs_[op.custom].tangent(nvec);
            break;
        }
        CU_CHECK(cudaGetLastError());
    }
    for (size_t k = 0; k < outputs.size(); k++) {
        const GNode &n = nodes_[outputs[k]];
        if (n.active && n.tan)
            CU_CHECK(cudaMemcpyAsync(results[k], n.tan.d(), sizeof(double) * n.size * nvec, cudaMemcpyDeviceToDevice,
                                     ex_.stream));
        else
            fill(ex_, results[k], n.size * nvec, 0.0);
    }
}

void Graph::vjp(const std::vector<int> &outputs, const std::vector<const double *> &seeds, int nvec,
                const std::vector<int> &inputs, const std::vector<double *> &results) {
    clear_derivatives();
    mark_active(inputs);
    for (size_t k = 0; k < outputs.size(); k++) {
        double *a = adjoint(outputs[k], nvec);
        axpby(ex_, nodes_[outputs[k]].size * nvec, 1.0, seeds[k], 1.0, a);
    }
    for (int oi = (int)ops_.size() - 1; oi >= 0; --oi) {
        const GOp &op = ops_[oi];
        if (!nodes_[op.out].active || !nodes_[op.out].adj) continue;
        Fp64Scope fp64(ex_, op.fp64);
        switch (op.kind) {
        case OpKind::Contract: {
            std::string s = op.spec;
            size_t comma = s.find(','), ar = s.find("->");
            std::string la = s.substr(0, comma), lb = s.substr(comma + 1, ar - comma - 1), lc = s.substr(ar + 2);
            TV cbar = tview(op.out, nvec, true);
            if (nodes_[op.a].active) {
                std::string sp = with_batch(lc) + "," + lb + "->" + with_batch(la);
                ccsd::contract(ex_, sp.c_str(), op.alpha, cbar, view(op.b), 1.0, tview(op.a, nvec, true));
            }
            if (nodes_[op.b].active) {
                std::string sp = la + "," + with_batch(lc) + "->" + with_batch(lb);
                ccsd::contract(ex_, sp.c_str(), op.alpha, view(op.a), cbar, 1.0, tview(op.b, nvec, true));
            }
            break;
        }
        case OpKind::Permute: {
            if (!nodes_[op.a].active) break;
            // a_bar[lin] += alpha * out_bar[lout]
            size_t ar = op.spec.find("->");
            std::string lin = op.spec.substr(0, ar) + BATCH, lout = op.spec.substr(ar + 2) + BATCH;
            TV obar = tview(op.out, nvec, true), abar = tview(op.a, nvec, true), pin;
            pin.p = obar.p;
            pin.nd = abar.nd;
            for (int k = 0; k < abar.nd; k++) {
                size_t pos = lout.find(lin[k]);
                pin.n[k] = obar.n[pos];
                pin.s[k] = obar.s[pos];
            }
            permute_add(ex_, op.alpha, pin, 1.0, abar);
            break;
        }
        case OpKind::Squareup:
            if (!nodes_[op.a].active) break;
            squareup_adj_kernel<<<grid_for(nov * (nov + 1) / 2 * nvec, 256), 256, 0, ex_.stream>>>(
                adjoint(op.out, nvec), adjoint(op.a, nvec), nov, nvec);
            ex_.launches++;
            break;
        case OpKind::PackHalf:
            if (!nodes_[op.a].active) break;
            pack_half_adj_kernel<<<grid_for(nov * (nov + 1) / 2 * nvec, 256), 256, 0, ex_.stream>>>(
                adjoint(op.out, nvec), adjoint(op.a, nvec), nov, nvec);
            ex_.launches++;
            break;
        case OpKind::PackSym:
            // d packed[(M, m)] / d F[x, y] = 1 for {x, y} = {M, m} (the diagonal's 1/2 meets two
            // equal entries): the adjoint is the full symmetric square-up of the packed adjoint
            if (!nodes_[op.a].active) break;
            squareup_batch_kernel<<<grid_for(nov * nov * nvec, 256), 256, 0, ex_.stream>>>(
                adjoint(op.out, nvec), adjoint(op.a, nvec), nov, nvec, 1);
            ex_.launches++;
            break;
        case OpKind::Trace: {
            if (!nodes_[op.a].active) break;
            const GNode &a = nodes_[op.a];
            trace_batch_kernel<<<grid_for(a.dims[0] * nvec, 128), 128, 0, ex_.stream>>>(
                adjoint(op.out, nvec), adjoint(op.a, nvec), a.dims[0], a.dims[1], nvec, 1);
            ex_.launches++;
            break;
        }
        case OpKind::Custom:
            customs_[op.custom].adjoint(nvec);
            break;
        }
        CU_CHECK(cudaGetLastError());
    }
    for (size_t k = 0; k < inputs.size(); k++) {
        const GNode &n = nodes_[inputs[k]];
        if (n.adj)
            CU_CHECK(cudaMemcpyAsync(results[k], n.adj.d(), sizeof(double) * n.size * nvec, cudaMemcpyDeviceToDevice,
                                     ex_.stream));
        else
            fill(ex_, results[k], n.size * nvec, 0.0);
    }
}

void pack_sym_add(Exec &ex, const double *full, double *packed, int64_t nov) {
    pack_sym_batch_kernel<<<grid_for(nov * (nov + 1) / 2, 256), 256, 0, ex.stream>>>(full, packed, nov, 1);
    ex.launches++;
    CU_CHECK(cudaGetLastError());
}

}  // namespace ccsd
