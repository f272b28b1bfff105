// planner.cpp -- gate lowering and the fusion planner (host, C++20).
//
// Lowering follows ket's gate definitions (src/simulator.cpp:38-254 for the
// matrices, :259-338 for the dispatch).  Planning replaces ket's Fuser
// (src/simulator.cpp:400-477):
//   * FUSE_NONE       one specialised kernel per gate (the plain method);
//   * FUSE_REFERENCE  ket's own rule -- a gate joins the open block only if
//                     its qubits are a subset of the block's first gate's;
//   * FUSE_GREEDY     blocks of up to k qubits grown over the gate DAG (a
//                     gate may join past gates on other qubits, never past a
//                     pending gate on one of its own qubits), kept only when a
//                     static byte model says one dense pass beats the
//                     specialised kernels it replaces;
//   * FUSE_LEARNED    the same candidate generator, with block costs from the
//                     MLP cost model and the partition chosen by predicted time.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <exception>
#include <numeric>
#include <string>
#include <thread>
#include <vector>

#include "internal.h"

namespace kb {

bool is_unitary(int type) { return type >= KETGPU_H && type <= KETGPU_CSWAP; }

int gate_arity(int type) {
  if (type < 0) return -1;
  if (type <= KETGPU_U) return 1;
  if (type <= KETGPU_SWAP) return 2;
  if (type <= KETGPU_CSWAP) return 3;
  return 0;
}

void validate_ops(int n, const ketgpu_op* ops, uint64_t nops) {
  for (uint64_t i = 0; i < nops; ++i) {
    const ketgpu_op& o = ops[i];
    if (o.type < 0 || o.type > KETGPU_PROBE)
      fail(KETGPU_ERR_INVALID, "ket: unknown gate code " + std::to_string(o.type));
    if (o.type == KETGPU_COMPOSITE)
      fail(KETGPU_ERR_INVALID, "ket: composite blocks must be flattened before the device call");
    const int a = is_unitary(o.type) ? gate_arity(o.type) : (o.type == KETGPU_MEASURE ? 1 : 0);
    for (int j = 0; j < a; ++j) {
      if (o.q[j] < 0 || o.q[j] >= n)
        fail(KETGPU_ERR_OUT_OF_RANGE, "ket: qubit index " + std::to_string(o.q[j]) +
                                          " is out of range for a " + std::to_string(n) +
                                          "-qubit circuit");
      for (int k = 0; k < j; ++k)
        if (o.q[j] == o.q[k])
          fail(KETGPU_ERR_INVALID,
               "ket: a gate cannot act on qubit " + std::to_string(o.q[j]) + " more than once");
    }
  }
}

void single_matrix(int type, const double* p, cplx m[4]) {
  const double r = 1.0 / std::sqrt(2.0);
  double c = 0, sn = 0;
  if (type == KETGPU_RX || type == KETGPU_RY || type == KETGPU_RZ || type == KETGPU_U ||
      type == KETGPU_CRX || type == KETGPU_CRY || type == KETGPU_CRZ || type == KETGPU_CU) {
    c = std::cos(p[0] / 2.0);
    sn = std::sin(p[0] / 2.0);
  }
  switch (type) {
    case KETGPU_H: case KETGPU_CH: m[0] = r; m[1] = r; m[2] = r; m[3] = -r; return;
    case KETGPU_X: case KETGPU_CX: case KETGPU_CCX: m[0] = 0; m[1] = 1; m[2] = 1; m[3] = 0; return;
    case KETGPU_Y: case KETGPU_CY: m[0] = 0; m[1] = cplx(0, -1); m[2] = cplx(0, 1); m[3] = 0; return;
    case KETGPU_Z: m[0] = 1; m[1] = 0; m[2] = 0; m[3] = -1; return;
    case KETGPU_S: m[0] = 1; m[1] = 0; m[2] = 0; m[3] = cplx(0, 1); return;
    case KETGPU_SDG: m[0] = 1; m[1] = 0; m[2] = 0; m[3] = cplx(0, -1); return;
    case KETGPU_T: m[0] = 1; m[1] = 0; m[2] = 0; m[3] = cplx(r, r); return;
    case KETGPU_TDG: m[0] = 1; m[1] = 0; m[2] = 0; m[3] = cplx(r, -r); return;
    case KETGPU_RX: case KETGPU_CRX:
      m[0] = c; m[1] = cplx(0, -sn); m[2] = cplx(0, -sn); m[3] = c; return;
    case KETGPU_RY: case KETGPU_CRY: m[0] = c; m[1] = -sn; m[2] = sn; m[3] = c; return;
    case KETGPU_RZ: case KETGPU_CRZ: m[0] = cplx(c, -sn); m[1] = 0; m[2] = 0; m[3] = cplx(c, sn); return;
    case KETGPU_U: case KETGPU_CU:
      m[0] = cplx(c, 0.0);
      m[1] = -std::polar(sn, p[2]);
      m[2] = std::polar(sn, p[1]);
      m[3] = std::polar(c, p[1] + p[2]);
      return;
    default:
      fail(KETGPU_ERR_LOGIC, "single_matrix: not a 1-qubit gate");
  }
}

namespace {

void set_fixed(Pass& p, std::initializer_list<int> qs) {
  p.nfixed = 0;
  for (int q : qs) p.fixed[p.nfixed++] = q;
  std::sort(p.fixed, p.fixed + p.nfixed);
}

}  // namespace

Pass lower_gate(const ketgpu_op& op) {
  Pass p;
  const int t = op.type;
  const auto bit = [&](int j) { return uint64_t{1} << op.q[j]; };
  if (gate_arity(t) == 1) {
    single_matrix(t, op.p, p.m);
    if (t == KETGPU_Z || t == KETGPU_S || t == KETGPU_SDG || t == KETGPU_T || t == KETGPU_TDG) {
      p.kind = PassKind::Phase;
      set_fixed(p, {op.q[0]});
      p.p0 = bit(0);
      p.m[0] = p.m[3];
    } else {
      p.kind = PassKind::Pair;
      set_fixed(p, {op.q[0]});
      p.p0 = 0;
      p.p1 = bit(0);
      p.mode = (t == KETGPU_X) ? kPairSwap : (t == KETGPU_RZ) ? kPairDiag : kPairGeneral;
    }
    return p;
  }
  switch (t) {
    case KETGPU_CZ: case KETGPU_CP:
      p.kind = PassKind::Phase;
      set_fixed(p, {op.q[0], op.q[1]});
      p.p0 = bit(0) | bit(1);
      p.m[0] = (t == KETGPU_CZ) ? cplx(-1.0, 0.0) : cplx(std::cos(op.p[0]), std::sin(op.p[0]));
      return p;
    case KETGPU_SWAP:
      p.kind = PassKind::Pair;
      p.mode = kPairSwap;
      set_fixed(p, {op.q[0], op.q[1]});
      p.p0 = bit(0);
      p.p1 = bit(1);
      return p;
    case KETGPU_CCX:
      p.kind = PassKind::Pair;
      p.mode = kPairSwap;
      set_fixed(p, {op.q[0], op.q[1], op.q[2]});
      p.p0 = bit(0) | bit(1);
      p.p1 = bit(0) | bit(1) | bit(2);
      return p;
    case KETGPU_CSWAP:
      p.kind = PassKind::Pair;
      p.mode = kPairSwap;
      set_fixed(p, {op.q[0], op.q[1], op.q[2]});
      p.p0 = bit(0) | bit(1);
      p.p1 = bit(0) | bit(2);
      return p;
    default: {  // controlled 2x2: CH, CX, CY, CRx, CRy, CRz, CU
      single_matrix(t, op.p, p.m);
      p.kind = PassKind::Pair;
      p.mode = (t == KETGPU_CX) ? kPairSwap : (t == KETGPU_CRZ) ? kPairDiag : kPairGeneral;
      set_fixed(p, {op.q[0], op.q[1]});
      p.p0 = bit(0);
      p.p1 = bit(0) | bit(1);
      return p;
    }
  }
}

double gate_traffic_fraction(const ketgpu_op& op) {
  const Pass p = lower_gate(op);
  if (p.kind == PassKind::Phase) return std::ldexp(1.0, -p.nfixed);
  return std::ldexp(1.0, 1 - p.nfixed);
}

namespace {

// Apply a lowered pass to a small dense vector (host, FP64).
void apply_small(const Pass& p, cplx* v, int nloc) {
  const uint64_t dim = uint64_t{1} << nloc;
  const uint64_t count = dim >> p.nfixed;
  for (uint64_t i = 0; i < count; ++i) {
    uint64_t b = i;
    for (int j = 0; j < p.nfixed; ++j) {
      const int f = p.fixed[j];
      b = ((b >> f) << (f + 1)) | (b & ((uint64_t{1} << f) - 1));
    }
    if (p.kind == PassKind::Phase) {
      v[b | p.p0] *= p.m[0];
      continue;
    }
    const cplx a = v[b | p.p0], c = v[b | p.p1];
    if (p.mode == kPairSwap) {
      v[b | p.p0] = c;
      v[b | p.p1] = a;
    } else {
      v[b | p.p0] = p.m[0] * a + p.m[1] * c;
      v[b | p.p1] = p.m[2] * a + p.m[3] * c;
    }
  }
}

}  // namespace

std::vector<cplx> block_matrix(const std::vector<const ketgpu_op*>& gates, const int* qubits, int k) {
  const int dim = 1 << k;
  std::vector<Pass> local;
  local.reserve(gates.size());
  for (const ketgpu_op* g : gates) {
    ketgpu_op o = *g;
    for (int j = 0; j < gate_arity(o.type); ++j) {
      int li = -1;
      for (int b = 0; b < k; ++b)
        if (qubits[b] == o.q[j]) li = b;
      if (li < 0) fail(KETGPU_ERR_LOGIC, "block_matrix: gate outside block");
      o.q[j] = li;
    }
    local.push_back(lower_gate(o));
  }
  std::vector<cplx> mat((size_t)dim * dim);
  std::vector<cplx> col(dim);
  for (int c = 0; c < dim; ++c) {
    std::fill(col.begin(), col.end(), cplx(0.0, 0.0));
    col[c] = 1.0;
    for (const Pass& p : local) apply_small(p, col.data(), k);
    for (int r = 0; r < dim; ++r) mat[(size_t)r * dim + c] = col[r];
  }
  return mat;
}

PlanOptions resolve_options(const ketgpu_options* opt) {
  PlanOptions o;
  if (!opt) return o;
  if (opt->precision != KETGPU_C64 && opt->precision != KETGPU_C128)
    fail(KETGPU_ERR_INVALID, "precision must be KETGPU_C64 or KETGPU_C128");
  if (opt->fusion < KETGPU_FUSE_NONE || opt->fusion > KETGPU_FUSE_LEARNED)
    fail(KETGPU_ERR_INVALID, "unknown fusion mode");
  o.precision = opt->precision;
  o.fusion = opt->fusion;
  // default block size: 6 qubits for complex64 on the tensor cores (their
  // 3xFP16 blocks stay memory-bound at k = 6, so fewer passes win), 5 for
  // the SIMT blocks, whose arithmetic grows with 2^k per amplitude
  o.max_k = opt->max_block_qubits ? opt->max_block_qubits
                                  : (opt->precision == KETGPU_C64 && opt->tensor_cores ? 6 : 5);
  if (o.max_k < 1 || o.max_k > 6) fail(KETGPU_ERR_INVALID, "max_block_qubits must be in [1, 6]");
  o.tensor = opt->tensor_cores != 0;
  o.renormalize = opt->renormalize;
  return o;
}

namespace {

struct Block {
  std::vector<int> gates;  // op indices, program order
  std::vector<int> qubits; // sorted
  bool diag = false;       // a run of diagonal gates: one Diagonal pass
};

uint64_t qubit_mask(const ketgpu_op& o) {
  uint64_t m = 0;
  for (int j = 0; j < gate_arity(o.type); ++j) m |= uint64_t{1} << o.q[j];
  return m;
}

// Cost (in full-state passes) of a dense k-qubit block pass: one HBM pass,
// plus the compute that outgrows it at large k.
double fused_cost_static(int k, int precision, bool tensor) {
  if (precision == KETGPU_C128) return k <= 4 ? 1.0 : (k == 5 ? 1.35 : 2.7);
  if (tensor && k >= 4 && k <= 6) return 1.0;
  return k <= 4 ? 1.0 : (k == 5 ? 1.45 : 2.9);
}

// Predicted gain (fraction of the greedy plan's predicted time) the learned
// planner needs before it departs from the greedy plan.
constexpr double kLearnedMargin = 0.02;

bool block_on_tensor_cores(int n, int k, const PlanOptions& opt) {
  return opt.precision == KETGPU_C64 && opt.tensor && tc_supported(k) && n >= k + 7;
}

// Greedy DAG-aware block growth over the gates `order` of `ops`.  With
// diag_runs, whenever the next gate to place is diagonal, every diagonal gate
// that can be moved to the front of what is left (no earlier non-diagonal
// gate shares a qubit with it) is collected; if that run spans more qubits
// than one block holds, it becomes a single Diagonal pass.
std::vector<Block> grow_blocks(int n, const ketgpu_op* ops, const std::vector<int>& order, int max_k,
                               bool diag_runs) {
  std::vector<Block> blocks;
  std::vector<char> done(order.size(), 0);
  size_t first = 0;
  std::vector<char> blocked(n, 0), inq(n, 0);
  const uint64_t all = n >= 64 ? ~uint64_t{0} : ((uint64_t{1} << n) - 1);
  while (true) {
    while (first < order.size() && done[first]) ++first;
    if (first == order.size()) break;
    if (diag_runs && is_diagonal_gate(ops[order[first]].type)) {
      std::vector<size_t> run;
      uint64_t blk = 0, span = 0;
      for (size_t i = first; i < order.size() && blk != all; ++i) {
        if (done[i]) continue;
        const ketgpu_op& o = ops[order[i]];
        const uint64_t m = qubit_mask(o);
        if (is_diagonal_gate(o.type) && !(m & blk)) {
          run.push_back(i);
          span |= m;
        } else {
          blk |= m;
        }
      }
      if (run.size() >= 2 && __builtin_popcountll(span) > max_k) {
        Block b;
        b.diag = true;
        for (size_t i : run) {
          done[i] = 1;
          b.gates.push_back(order[i]);
        }
        for (int q = 0; q < n; ++q)
          if ((span >> q) & 1) b.qubits.push_back(q);
        blocks.push_back(std::move(b));
        continue;
      }
    }
    Block b;
    std::fill(blocked.begin(), blocked.end(), 0);
    std::fill(inq.begin(), inq.end(), 0);
    int nq = 0, nblocked = 0;
    for (size_t i = first; i < order.size(); ++i) {
      if (done[i]) continue;
      const ketgpu_op& o = ops[order[i]];
      const int a = gate_arity(o.type);
      bool hit = false;
      int add = 0;
      for (int j = 0; j < a; ++j) {
        if (blocked[o.q[j]]) hit = true;
        if (!inq[o.q[j]]) ++add;
      }
      if (b.gates.empty() || (!hit && nq + add <= max_k)) {
        for (int j = 0; j < a; ++j)
          if (!inq[o.q[j]]) {
            inq[o.q[j]] = 1;
            ++nq;
          }
        b.gates.push_back((int)i);
        done[i] = 1;
      } else {
        for (int j = 0; j < a; ++j)
          if (!blocked[o.q[j]]) {
            blocked[o.q[j]] = 1;
            ++nblocked;
          }
        if (nblocked == n) break;
        // nothing more can join once every block qubit is blocked and the
        // block is full
        if (nq == max_k) {
          bool open = false;
          for (int q = 0; q < n; ++q)
            if (inq[q] && !blocked[q]) open = true;
          if (!open) break;
        }
      }
    }
    for (int q = 0; q < n; ++q)
      if (inq[q]) b.qubits.push_back(q);
    for (int& gi : b.gates) gi = order[gi];
    blocks.push_back(std::move(b));
  }
  return blocks;
}

// Topological orders of a segment's gates for the greedy block growth.  The
// program order is one; a "band" order of width w sorts the gates by
// ((ASAP depth + offset) / w, lowest qubit, depth), subject to every dependency, so
// growth from the first gate follows a few neighbouring qubits through w
// levels of the circuit before moving on: light-cone-shaped blocks.  On the
// 30-qubit, 40-layer brick wall at k = 5 the best band order needs 119
// passes against 154 in program order.  Returns op indices.
std::vector<int> band_order(const ketgpu_op* ops, const std::vector<int>& seg, int n, int w, int off) {
  const size_t G = seg.size();
  std::vector<int> depth(G, 0), indeg(G, 0), qmin(G, 0), last(n, -1);
  std::vector<std::vector<int>> succ(G);
  for (size_t i = 0; i < G; ++i) {
    const ketgpu_op& o = ops[seg[i]];
    int d = 0, lo = n;
    for (int j = 0; j < gate_arity(o.type); ++j) {
      const int q = o.q[j];
      lo = std::min(lo, q);
      if (last[q] >= 0) {
        d = std::max(d, depth[last[q]] + 1);
        succ[last[q]].push_back((int)i);
        ++indeg[i];
      }
      last[q] = (int)i;
    }
    depth[i] = d;
    qmin[i] = lo;
  }
  auto later = [&](int a, int b) {  // heap order: the smallest key first
    const int ba = (depth[a] + off) / w, bb = (depth[b] + off) / w;
    if (ba != bb) return ba > bb;
    if (qmin[a] != qmin[b]) return qmin[a] > qmin[b];
    if (depth[a] != depth[b]) return depth[a] > depth[b];
    return a > b;
  };
  std::vector<int> heap, out;
  out.reserve(G);
  for (size_t i = 0; i < G; ++i)
    if (!indeg[i]) heap.push_back((int)i);
  std::make_heap(heap.begin(), heap.end(), later);
  while (!heap.empty()) {
    std::pop_heap(heap.begin(), heap.end(), later);
    const int i = heap.back();
    heap.pop_back();
    out.push_back(seg[i]);
    for (int sidx : succ[i])
      if (--indeg[sidx] == 0) {
        heap.push_back(sidx);
        std::push_heap(heap.begin(), heap.end(), later);
      }
  }
  return out;
}

// Band widths the planner tries besides the program order, each at every
// offset (the band boundaries shifted by 0 .. w-1 levels).
constexpr int kBandWidths[] = {3, 4, 5, 6, 7, 8};

// Static cost of a partition in full-state passes: each block fused or as
// its separate gates, whichever is cheaper; a diagonal run is one pass.
double partition_cost(const ketgpu_op* ops, const std::vector<Block>& blocks, const PlanOptions& opt) {
  double total = 0;
  for (const Block& b : blocks) {
    if (b.diag) {
      total += 1.0;
      continue;
    }
    double separate = 0;
    for (int gi : b.gates) separate += gate_traffic_fraction(ops[gi]);
    total += b.gates.size() > 1 ? std::min(separate, fused_cost_static((int)b.qubits.size(), opt.precision,
                                                                         opt.tensor))
                                : separate;
  }
  return total;
}

// Greedy growth over the program order and every band order (width,
// offset); the partition with the least static cost, the earliest candidate
// on ties.  The candidates are grown on up to 16 host threads.
std::vector<Block> best_partition(int n, const ketgpu_op* ops, const std::vector<int>& seg,
                                  const PlanOptions& opt) {
  std::vector<std::pair<int, int>> cands{{0, 0}};  // (0, 0): the program order
  for (int w : kBandWidths)
    for (int off = 0; off < w; ++off) cands.push_back({w, off});
  const size_t C = cands.size();
  std::vector<std::vector<Block>> parts(C);
  std::vector<double> cost(C, 0.0);
  auto work = [&](size_t c) {
    const std::vector<int> order = cands[c].first ? band_order(ops, seg, n, cands[c].first, cands[c].second) : seg;
    parts[c] = grow_blocks(n, ops, order, std::max(1, opt.max_k), true);
    cost[c] = partition_cost(ops, parts[c], opt);
  };
  const unsigned nt = seg.size() < 256 ? 1u : std::min<unsigned>(16u, std::max(1u, std::thread::hardware_concurrency()));
  if (nt <= 1) {
    for (size_t c = 0; c < C; ++c) work(c);
  } else {
    std::atomic<size_t> next{0};
    std::vector<std::thread> th;
    for (unsigned t = 0; t < nt; ++t)
      th.emplace_back([&] {
        for (size_t c; (c = next.fetch_add(1)) < C;) work(c);
      });
    for (auto& x : th) x.join();
  }
  size_t best = 0;
  for (size_t c = 1; c < C; ++c)
    if (cost[c] < cost[best] - 1e-9) best = c;
  return std::move(parts[best]);
}

// ket's Fuser block rule on one barrier-free segment.
std::vector<Block> reference_blocks(const ketgpu_op* ops, const std::vector<int>& order) {
  std::vector<Block> blocks;
  Block cur;
  std::vector<int> first_qubits;
  for (int idx : order) {
    const ketgpu_op& o = ops[idx];
    const int a = gate_arity(o.type);
    bool subset = !cur.gates.empty();
    for (int j = 0; j < a && subset; ++j)
      if (std::find(first_qubits.begin(), first_qubits.end(), o.q[j]) == first_qubits.end()) subset = false;
    if (!cur.gates.empty() && !subset) {
      blocks.push_back(std::move(cur));
      cur = Block();
    }
    if (cur.gates.empty()) {
      first_qubits.assign(o.q, o.q + a);
      cur.qubits = first_qubits;
    }
    cur.gates.push_back(idx);
  }
  if (!cur.gates.empty()) blocks.push_back(std::move(cur));
  return blocks;
}

void emit_single(Plan& plan, const ketgpu_op& o, int idx) {
  Pass p = lower_gate(o);
  p.first_op = idx;
  p.n_gates = 1;
  p.gates = {idx};
  plan.passes.push_back(p);
}

void emit_run(Plan& plan, const ketgpu_op* ops, const std::vector<int>& gates) {
  std::vector<Pass> lowered;
  for (int gi : gates) lowered.push_back(lower_gate(ops[gi]));
  Pass p;
  p.kind = PassKind::SharedRun;
  p.run_index = plan.runs.size();
  p.first_op = gates.front();
  p.n_gates = (int)gates.size();
  p.gates = gates;
  plan.runs.push_back(std::move(lowered));
  plan.passes.push_back(p);
}

void emit_diagonal(Plan& plan, int n, const ketgpu_op* ops, const Block& b) {
  DiagPoly poly;
  poly.a.assign(n, 0.0);
  poly.b.assign((size_t)n * n, 0.0);
  for (int gi : b.gates) add_diagonal_gate(ops[gi], poly, n);
  Pass p;
  p.kind = PassKind::Diagonal;
  p.k = (int)b.qubits.size();
  p.diag_index = plan.diags.size();
  p.first_op = b.gates.front();
  p.n_gates = (int)b.gates.size();
  p.gates = b.gates;
  plan.diags.push_back(std::move(poly));
  plan.passes.push_back(p);
}

// Block matrices of the plan being built on this thread: emit_fused records
// each one as a job and build_plan computes them all at the end, in
// parallel (at k = 6 they are most of the planning time).
struct MatrixJob {
  size_t index;
  std::vector<int> gates;
  std::vector<int> qubits;
};
thread_local std::vector<MatrixJob>* t_matrix_jobs = nullptr;

void compute_matrices(Plan& plan, const ketgpu_op* ops, const std::vector<MatrixJob>& jobs) {
  auto work = [&](const MatrixJob& jb) {
    std::vector<const ketgpu_op*> gs;
    for (int gi : jb.gates) gs.push_back(&ops[gi]);
    plan.matrices[jb.index] = block_matrix(gs, jb.qubits.data(), (int)jb.qubits.size());
  };
  const unsigned nt = jobs.size() < 16 ? 1u
                      : std::min<unsigned>(16u, std::max(1u, std::thread::hardware_concurrency()));
  if (nt <= 1) {
    for (const MatrixJob& jb : jobs) work(jb);
    return;
  }
  std::atomic<size_t> next{0};
  std::exception_ptr err;
  std::atomic<bool> failed{false};
  std::vector<std::thread> th;
  for (unsigned t = 0; t < nt; ++t)
    th.emplace_back([&] {
      for (size_t i; (i = next.fetch_add(1)) < jobs.size();) {
        try {
          work(jobs[i]);
        } catch (...) {
          if (!failed.exchange(true)) err = std::current_exception();
        }
      }
    });
  for (auto& x : th) x.join();
  if (err) std::rethrow_exception(err);
}

void emit_fused(Plan& plan, int n, const ketgpu_op* ops, const Block& b, const PlanOptions& opt) {
  std::vector<const ketgpu_op*> gs;
  for (int gi : b.gates) gs.push_back(&ops[gi]);
  std::vector<int> qs = b.qubits;
  std::sort(qs.begin(), qs.end());
  // complex64 on the tensor cores: a 2- or 3-qubit block is padded to 4
  // qubits (identity on the highest free qubits, so the block's group bits
  // stay low) and runs at HBM speed instead of on the SIMT block kernel.
  if (qs.size() >= 2 && qs.size() < 4 && !block_on_tensor_cores(n, (int)qs.size(), opt) &&
      block_on_tensor_cores(n, 4, opt)) {
    for (int q = n - 1; q >= 0 && qs.size() < 4; --q)
      if (std::find(qs.begin(), qs.end(), q) == qs.end()) qs.push_back(q);
    std::sort(qs.begin(), qs.end());
  }
  const int k = (int)qs.size();
  Pass p;
  p.first_op = b.gates.front();
  p.n_gates = (int)b.gates.size();
  p.gates = b.gates;
  if (k == 1) {  // one 2x2 through the streaming pair kernel
    const std::vector<cplx> mat = block_matrix(gs, qs.data(), k);
    p.kind = PassKind::Pair;
    p.mode = kPairGeneral;
    p.nfixed = 1;
    p.fixed[0] = qs[0];
    p.p0 = 0;
    p.p1 = uint64_t{1} << qs[0];
    for (int j = 0; j < 4; ++j) p.m[j] = mat[j];
    plan.passes.push_back(p);
    return;
  }
  p.kind = PassKind::Fused;
  p.k = k;
  for (int j = 0; j < k; ++j) p.qubits[j] = qs[j];
  p.tensor = block_on_tensor_cores(n, k, opt);
  p.mat_index = plan.matrices.size();
  if (t_matrix_jobs) {
    plan.matrices.emplace_back();
    t_matrix_jobs->push_back({p.mat_index, b.gates, qs});
  } else {
    plan.matrices.push_back(block_matrix(gs, qs.data(), k));
  }
  plan.passes.push_back(p);
}

}  // namespace

// 48 features: scale (n, bytes), pass kind, block geometry (k, span, low /
// high qubits, runs of adjacent qubits, coalescing), gate content (counts by
// kind), precision and an L2-residency flag.  Index layout is fixed; the
// trained cost model depends on it.
void pass_features(int n, int precision, const std::vector<const ketgpu_op*>& gates,
                   const std::vector<int>& qubits, bool fused, bool tensor, float* f) {
  for (int i = 0; i < kFeatures; ++i) f[i] = 0.f;
  const double amp = precision == KETGPU_C64 ? 8.0 : 16.0;
  const double state = amp * std::ldexp(1.0, n);
  double frac = 1.0;
  if (!fused && gates.size() == 1) frac = gate_traffic_fraction(*gates[0]);
  const int k = (int)qubits.size();
  int lo = n, hi = -1, runs = 0, low7 = 0;
  std::vector<int> qs = qubits;
  std::sort(qs.begin(), qs.end());
  for (size_t i = 0; i < qs.size(); ++i) {
    lo = std::min(lo, qs[i]);
    hi = std::max(hi, qs[i]);
    if (i == 0 || qs[i] != qs[i - 1] + 1) ++runs;
    if (qs[i] < 7) ++low7;
  }
  f[0] = (float)n / 32.f;
  f[1] = (float)(std::log2(2.0 * state * frac) / 40.0);
  f[2] = fused ? 1.f : 0.f;
  f[3] = tensor ? 1.f : 0.f;
  f[4] = (float)k / 6.f;
  f[5] = (float)gates.size() / 64.f;
  f[6] = k ? (float)lo / (float)n : 0.f;
  f[7] = k ? (float)hi / (float)n : 0.f;
  f[8] = k ? (float)(hi - lo + 1) / (float)n : 0.f;
  f[9] = (k && lo == 0) ? 1.f : 0.f;
  f[10] = (float)low7 / 6.f;
  f[11] = (float)runs / 6.f;
  f[12] = (float)frac;
  f[13] = precision == KETGPU_C128 ? 1.f : 0.f;
  if (k >= 1 && k <= 6) f[13 + k] = 1.f;  // 14..19
  for (const ketgpu_op* g : gates) {
    int slot;
    switch (g->type) {
      case KETGPU_H: slot = 0; break;
      case KETGPU_S: case KETGPU_SDG: case KETGPU_Z: case KETGPU_T: case KETGPU_TDG: slot = 1; break;
      case KETGPU_RX: slot = 2; break;
      case KETGPU_RY: slot = 3; break;
      case KETGPU_RZ: slot = 4; break;
      case KETGPU_U: case KETGPU_X: case KETGPU_Y: slot = 5; break;
      case KETGPU_CX: case KETGPU_CY: slot = 6; break;
      case KETGPU_CZ: slot = 7; break;
      case KETGPU_CP: slot = 8; break;
      case KETGPU_CRX: case KETGPU_CRY: case KETGPU_CRZ: case KETGPU_CU: case KETGPU_CH: slot = 9; break;
      case KETGPU_SWAP: slot = 10; break;
      case KETGPU_CCX: slot = 11; break;
      case KETGPU_CSWAP: slot = 12; break;
      default: slot = 13; break;
    }
    f[20 + slot] += 1.f / 16.f;  // 20..33
  }
  for (int q : qs) {
    if (q < 8) f[34 + q] = 1.f;                    // 34..41
    if (q >= n - 4) f[42 + (n - 1 - q)] = 1.f;      // 42..45
  }
  f[46] = state <= 126e6 ? 1.f : 0.f;
  f[47] = 1.f;
}

void build_plan(Plan& plan, int n, const ketgpu_op* ops, uint64_t nops, const PlanOptions& opt) {
  plan.n = n;
  plan.precision = opt.precision;
  plan.ops.assign(ops, ops + nops);
  plan.passes.clear();
  plan.matrices.clear();
  std::vector<MatrixJob> jobs;
  struct JobScope {
    explicit JobScope(std::vector<MatrixJob>* j) { t_matrix_jobs = j; }
    ~JobScope() { t_matrix_jobs = nullptr; }
  } job_scope(&jobs);
  uint64_t n_gates = 0;
  double predicted = 0;
  const size_t amp = opt.precision == KETGPU_C64 ? 8 : 16;
  // Split at structural ops: they are fusion barriers (simulator.cpp:496).
  std::vector<int> seg;
  auto flush = [&]() {
    if (seg.empty()) return;
    if (opt.fusion == KETGPU_FUSE_NONE) {
      // One kernel per gate, except that consecutive gates on qubits below
      // kRunBits are staged through shared memory as one pass.
      const int bits = std::min(n, kRunBits);
      size_t i = 0;
      while (i < seg.size()) {
        size_t j = i;
        while (j < seg.size() && j - i < (size_t)kRunMaxGates && (qubit_mask(ops[seg[j]]) >> bits) == 0) ++j;
        if (j - i >= 2) {
          emit_run(plan, ops, std::vector<int>(seg.begin() + i, seg.begin() + j));
          i = j;
        } else {
          emit_single(plan, ops[seg[i]], seg[i]);
          ++i;
        }
      }
    } else if (opt.fusion == KETGPU_FUSE_REFERENCE) {
      for (const Block& b : reference_blocks(ops, seg)) {
        if (b.gates.size() == 1) emit_single(plan, ops[b.gates[0]], b.gates[0]);
        else emit_fused(plan, n, ops, b, opt);
      }
    } else if (opt.fusion == KETGPU_FUSE_LEARNED && learned_model_attached()) {
      // Candidate partitions (greedy growth at k = 3..6); every block scored
      // fused and as its separate gates by the cost model in one batched
      // inference; the partition with the least predicted time wins, each
      // block taking its cheaper form.
      const int kmin_cand = std::min(3, std::max(1, opt.max_k));
      const int kmax_cap = std::max(kmin_cand, std::min(6, opt.max_k + 1));
      // per k: the greedy partition of least static cost over the program
      // order and the band orders (what FUSE_GREEDY would emit at that k)
      std::vector<std::vector<Block>> cands;
      for (int kc = kmin_cand; kc <= kmax_cap; ++kc) {
        PlanOptions ok = opt;
        ok.max_k = kc;
        cands.push_back(best_partition(n, ops, seg, ok));
      }
      std::vector<float> rows;
      float fr[kFeatures];
      // single-gate rows, one per gate of the segment
      std::vector<size_t> single_row(nops, 0);
      for (int gi : seg) {
        std::vector<int> q1(ops[gi].q, ops[gi].q + gate_arity(ops[gi].type));
        pass_features(n, opt.precision, {&ops[gi]}, q1, false, false, fr);
        single_row[gi] = rows.size() / kFeatures;
        rows.insert(rows.end(), fr, fr + kFeatures);
      }
      std::vector<std::vector<size_t>> fused_row(cands.size());
      for (size_t c = 0; c < cands.size(); ++c)
        for (const Block& b : cands[c]) {
          if (b.diag) {
            // A Diagonal pass streams the whole state once: scored as the
            // model's time of a dense one-qubit pass on the run's top qubit.
            ketgpu_op proxy{};
            proxy.type = KETGPU_U;
            proxy.nq = 1;
            proxy.q[0] = b.qubits.back();
            pass_features(n, opt.precision, {&proxy}, {proxy.q[0]}, false, false, fr);
            fused_row[c].push_back(rows.size() / kFeatures);
            rows.insert(rows.end(), fr, fr + kFeatures);
            continue;
          }
          std::vector<const ketgpu_op*> gs;
          for (int gi : b.gates) gs.push_back(&ops[gi]);
          pass_features(n, opt.precision, gs, b.qubits, true,
                        block_on_tensor_cores(n, (int)b.qubits.size(), opt), fr);
          fused_row[c].push_back(rows.size() / kFeatures);
          rows.insert(rows.end(), fr, fr + kFeatures);
        }
      std::vector<float> us;
      learned_predict(rows, us);
      size_t best = 0;
      double best_t = 1e300;
      std::vector<std::vector<char>> choice(cands.size());
      for (size_t c = 0; c < cands.size(); ++c) {
        double tot = 0;
        for (size_t bi = 0; bi < cands[c].size(); ++bi) {
          const Block& b = cands[c][bi];
          if (b.diag) {
            choice[c].push_back(2);
            tot += us[fused_row[c][bi]];
            continue;
          }
          double sep = 0;
          for (int gi : b.gates) sep += us[single_row[gi]];
          const double fu = us[fused_row[c][bi]];
          const bool fuse = b.gates.size() > 1 && fu < sep;
          choice[c].push_back(fuse ? 1 : 0);
          tot += fuse ? fu : sep;
        }
        if (tot < best_t) {
          best_t = tot;
          best = c;
        }
      }
      // The greedy plan (growth at max_k, static fuse rule), scored by the
      // same model: the learned choice replaces it only when the model
      // predicts a clear gain, so model error on near-equal plans cannot
      // make the learned plan slower than greedy.
      const size_t gk = (size_t)(std::max(kmin_cand, std::min(opt.max_k, kmax_cap)) - kmin_cand);
      double greedy_t = 0;
      std::vector<char> greedy_choice;
      for (size_t bi = 0; bi < cands[gk].size(); ++bi) {
        const Block& b = cands[gk][bi];
        char ch;
        if (b.diag) {
          ch = 2;
          greedy_t += us[fused_row[gk][bi]];
        } else {
          double sep = 0, frac = 0;
          for (int gi : b.gates) {
            sep += us[single_row[gi]];
            frac += gate_traffic_fraction(ops[gi]);
          }
          ch = b.gates.size() > 1 && fused_cost_static((int)b.qubits.size(), opt.precision, opt.tensor) < frac;
          greedy_t += ch ? us[fused_row[gk][bi]] : sep;
        }
        greedy_choice.push_back(ch);
      }
      if (!(best_t < (1.0 - kLearnedMargin) * greedy_t)) {
        best = gk;
        best_t = greedy_t;
        choice[gk] = greedy_choice;
      }
      predicted += best_t;
      for (size_t bi = 0; bi < cands[best].size(); ++bi) {
        const Block& b = cands[best][bi];
        if (choice[best][bi] == 2) emit_diagonal(plan, n, ops, b);
        else if (choice[best][bi]) emit_fused(plan, n, ops, b, opt);
        else
          for (int gi : b.gates) emit_single(plan, ops[gi], gi);
      }
    } else {
      // greedy growth over the program order and every band order; the
      // partition with the least static cost wins (the program order on ties)
      std::vector<Block> best = best_partition(n, ops, seg, opt);
      for (const Block& b : best) {
        if (b.diag) {
          emit_diagonal(plan, n, ops, b);
          continue;
        }
        if (b.gates.size() == 1) {
          emit_single(plan, ops[b.gates[0]], b.gates[0]);
          continue;
        }
        const int k = (int)b.qubits.size();
        double separate = 0;
        for (int gi : b.gates) separate += gate_traffic_fraction(ops[gi]);
        if (fused_cost_static(k, opt.precision, opt.tensor) < separate) {
          emit_fused(plan, n, ops, b, opt);
        } else {
          for (int gi : b.gates) emit_single(plan, ops[gi], gi);
        }
      }
    }
    seg.clear();
  };
  for (uint64_t i = 0; i < nops; ++i) {
    if (is_unitary(ops[i].type)) {
      seg.push_back((int)i);
      ++n_gates;
    } else {
      flush();
    }
  }
  flush();
  t_matrix_jobs = nullptr;
  compute_matrices(plan, ops, jobs);
  bool any_tensor = false;
  for (const Pass& p : plan.passes) any_tensor |= p.tensor;
  if ((opt.renormalize == 0 && any_tensor) || (opt.renormalize > 0 && !plan.passes.empty())) {
    Pass cap, res;
    cap.kind = PassKind::NormCapture;
    res.kind = PassKind::NormRestore;
    // a tensor-core block right before the restore sums the norm as it stores
    if (!plan.passes.empty() && plan.passes.back().kind == PassKind::Fused && plan.passes.back().tensor) {
      plan.passes.back().norm_out = true;
      res.norm_out = true;
    }
    plan.passes.insert(plan.passes.begin(), cap);
    plan.passes.push_back(res);
  }
  ketgpu_plan_stats& st = plan.stats;
  st = ketgpu_plan_stats{};
  st.n_gates = n_gates;
  st.n_passes = plan.passes.size();
  for (const Pass& p : plan.passes) {
    st.bytes += p.bytes(n, amp);
    if (p.kind == PassKind::Fused) {
      ++st.n_fused;
      if (p.tensor) ++st.n_tensor;
      st.flops += 8.0 * (double)(1 << p.k) * (double)(uint64_t{1} << n);
    }
  }
  st.predicted_us = predicted;
}

}  // namespace kb
