// partition.cpp -- element partition and halo lists (see partition.h).  The
// reference decomposes with METIS through adcprep and exchanges ghost
// elements with MPI (messenger_elem.F); here a partition is a contiguous
// range of the Morton order, and the halo is derived from the edge graph.
#include "partition.h"

#include <algorithm>
#include <parallel/algorithm>
#include <cstdint>
#include <string>

#include "abi_util.h"

namespace dgswem {

std::vector<int> morton_order(const std::vector<double>& px, const std::vector<double>& py,
                              const std::vector<int>& group) {
  const int n = (int)px.size();
  const bool grouped = !group.empty();
  int ng = 1;
  if (grouped)
    for (int i = 0; i < n; ++i) ng = std::max(ng, group[i] + 1);
  // bounding box of each group
  std::vector<double> x0(ng, 1e300), x1(ng, -1e300), y0(ng, 1e300), y1(ng, -1e300);
  for (int i = 0; i < n; ++i) {
    const int g = grouped ? group[i] : 0;
    x0[g] = std::min(x0[g], px[i]); x1[g] = std::max(x1[g], px[i]);
    y0[g] = std::min(y0[g], py[i]); y1[g] = std::max(y1[g], py[i]);
  }
  auto spread = [](uint64_t v) {  // bits of v at the even positions
    uint64_t r = 0;
    for (int b = 0; b < 21; ++b) r |= ((v >> b) & 1u) << (2 * b);
    return r;
  };
  std::vector<uint64_t> key(n);
#pragma omp parallel for schedule(static)
  for (int i = 0; i < n; ++i) {
    const int g = grouped ? group[i] : 0;
    const double span = std::max(std::max(x1[g] - x0[g], y1[g] - y0[g]), 1e-300);
    const double scale = (double)((1u << 21) - 1) / span;
    const uint64_t ix = (uint64_t)((px[i] - x0[g]) * scale), iy = (uint64_t)((py[i] - y0[g]) * scale);
    key[i] = spread(ix) | spread(iy) << 1;
  }
  std::vector<int> perm(n);
  for (int i = 0; i < n; ++i) perm[i] = i;
  // (group, key, index) is a strict total order, so the parallel sort gives
  // the stable sort's permutation
  __gnu_parallel::sort(perm.begin(), perm.end(), [&](int a, int b) {
    const int ga = grouped ? group[a] : 0, gb = grouped ? group[b] : 0;
    if (ga != gb) return ga < gb;
    if (key[a] != key[b]) return key[a] < key[b];
    return a < b;
  });
  return perm;
}

void validate_mesh_ids(const dgswem_cuda_setup* s) {
  auto need = [](bool ok, const char* what) {
    if (!ok) throw Failure(DGSWEM_ERR_ARG, what);
  };
  need(s->nm && s->neled && s->nedel && s->nedsd, "setup lacks mesh arrays");
  const size_t ne = (size_t)s->ne, ned = (size_t)s->nedges;
  for (size_t i = 0; i < 3 * ne; ++i) {
    need(s->nm[i] >= 1 && s->nm[i] <= s->np, "NM refers to a node outside 1..NP");
    need(s->neled[i] >= 1 && (size_t)s->neled[i] <= ned, "NELED refers to an edge outside 1..NEDGES");
  }
  for (size_t k = 0; k < 2 * ned; ++k) {
    need(s->nedel[k] >= 0 && s->nedel[k] <= s->ne, "NEDEL refers to an element outside 0..NE");
    if (s->nedel[k] != 0) need(s->nedsd[k] >= 1 && s->nedsd[k] <= 3, "NEDSD is not a local edge number 1..3");
  }
  const struct { const int* list; int n; const char* what; } lists[] = {
      {s->needn, s->needs, "NEEDN"}, {s->nledn, s->nleds, "NLEDN"}, {s->nfedn, s->nfeds, "NFEDN"},
      {s->nredn, s->nreds, "NREDN"}, {s->nebsegn, s->nebseg, "NEBSEGN"}, {s->nibsegn, 2 * s->nibseg, "NIBSEGN"}};
  for (const auto& L : lists) {
    if (L.n <= 0) continue;
    if (!L.list) throw Failure(DGSWEM_ERR_ARG, std::string("setup lacks ") + L.what);
    for (int i = 0; i < L.n; ++i)  // NIBSEGN's opposite edge may be 0 (no partner)
      if (!(L.list[i] >= 1 && (size_t)L.list[i] <= ned) && !(L.list == s->nibsegn && i % 2 == 1 && L.list[i] == 0))
        throw Failure(DGSWEM_ERR_ARG, std::string(L.what) + " refers to an edge outside 1..NEDGES");
  }
}

std::vector<int> mesh_components(const dgswem_cuda_setup* s, std::vector<int>* node_comp) {
  const int ne = s->ne, np = s->np;
  std::vector<int> parent(np);
  for (int i = 0; i < np; ++i) parent[i] = i;
  auto find = [&](int a) {
    while (parent[a] != a) a = parent[a] = parent[parent[a]];
    return a;
  };
  for (int e = 0; e < ne; ++e) {
    const int a = find(s->nm[e] - 1);
    for (int v = 1; v < 3; ++v) {
      const int b = find(s->nm[e + (size_t)ne * v] - 1);
      if (a != b) parent[b] = a;
    }
  }
  // components numbered by their first element in input order
  std::vector<int> label(np, -1), elem(ne);
  int nc = 0;
  for (int e = 0; e < ne; ++e) {
    const int r = find(s->nm[e] - 1);
    if (label[r] < 0) label[r] = nc++;
    elem[e] = label[r];
  }
  if (node_comp) {
    node_comp->assign(np, 0);
    for (int i = 0; i < np; ++i) {
      const int r = find(i);
      (*node_comp)[i] = label[r] < 0 ? 0 : label[r];  // a node in no element: any group
    }
  }
  return elem;
}

PartPlan make_part_plan(const dgswem_cuda_setup* s, int part, int nparts) {
  const int ne = s->ne, np = s->np;
  if (nparts < 1 || part < 0 || part >= nparts) throw Failure(DGSWEM_ERR_ARG, "partition index out of range");
  if (nparts > ne) throw Failure(DGSWEM_ERR_ARG, "more partitions than elements");
  PartPlan P;
  P.part = part;
  P.nparts = nparts;
  {
    std::vector<double> cx(ne), cy(ne);
    for (int e = 0; e < ne; ++e) {
      double sx = 0.0, sy = 0.0;
      for (int v = 0; v < 3; ++v) {
        const int n = s->nm[e + (size_t)ne * v] - 1;
        if (n < 0 || n >= np) throw Failure(DGSWEM_ERR_ARG, "NM refers to a node outside 1..NP");
        sx += s->x[n];
        sy += s->y[n];
      }
      cx[e] = sx / 3.0;
      cy[e] = sy / 3.0;
    }
    P.order = morton_order(cx, cy, mesh_components(s, nullptr));
  }
  std::vector<int> pos(ne);
  for (int i = 0; i < ne; ++i) pos[P.order[i]] = i;
  P.owner.assign(ne, 0);
  for (int q = 0; q < nparts; ++q) {
    const long lo = (long)q * ne / nparts, hi = (long)(q + 1) * ne / nparts;
    for (long i = lo; i < hi; ++i) P.owner[P.order[i]] = q;
  }
  P.send[0].assign(nparts, {});
  P.send[1].assign(nparts, {});
  P.recv[0].assign(nparts, {});
  P.recv[1].assign(nparts, {});
  const long lo = (long)part * ne / nparts, hi = (long)(part + 1) * ne / nparts;
  P.n_own = (int)(hi - lo);
  P.local.assign(P.order.begin() + lo, P.order.begin() + hi);
  if (nparts == 1) return P;
  // adjacency: edges (NEDEL of the interior edges), barrier partners, node stars
  std::vector<std::vector<int>> full_nb(ne);
  for (int g = 0; g < s->nedges; ++g) {
    const int a = s->nedel[2 * (size_t)g], b = s->nedel[2 * (size_t)g + 1];
    if (a != 0 && b != 0) {
      full_nb[a - 1].push_back(b - 1);
      full_nb[b - 1].push_back(a - 1);
    }
  }
  for (int L = 0; L < s->nibseg; ++L) {
    const int gb = s->nibsegn[2 * L], gf = s->nibsegn[2 * L + 1];
    if (gb == 0 || gf == 0) continue;
    const int eb = s->nedel[2 * (size_t)(gb - 1)] - 1, ef = s->nedel[2 * (size_t)(gf - 1)] - 1;
    if (eb < 0 || ef < 0) continue;
    full_nb[eb].push_back(ef);
    full_nb[ef].push_back(eb);
  }
  std::vector<int> sp(np + 1, 0), st(3 * (size_t)ne);
  for (int e = 0; e < ne; ++e)
    for (int v = 0; v < 3; ++v) ++sp[s->nm[e + (size_t)ne * v]];
  for (int n = 0; n < np; ++n) sp[n + 1] += sp[n];
  {
    std::vector<int> cur(sp.begin(), sp.end() - 1);
    for (int e = 0; e < ne; ++e)
      for (int v = 0; v < 3; ++v) st[cur[s->nm[e + (size_t)ne * v] - 1]++] = e;
  }
  std::vector<char> ghost_kind(ne, 0);  // bit k: a halo of kind k
  for (long i = lo; i < hi; ++i) {
    const int e = P.order[i];
    std::vector<char> sent_to(2 * (size_t)nparts, 0);
    for (int nb : full_nb[e]) {
      const int q = P.owner[nb];
      if (q == part) continue;
      ghost_kind[nb] |= 2;
      if (!sent_to[2 * q + 1]) { P.send[kHaloFull][q].push_back(e); sent_to[2 * q + 1] = 1; }
    }
    for (int v = 0; v < 3; ++v) {
      const int n = s->nm[e + (size_t)ne * v] - 1;
      for (int k = sp[n]; k < sp[n + 1]; ++k) {
        const int nb = st[k];
        const int q = P.owner[nb];
        if (q == part) continue;
        ghost_kind[nb] |= 1;
        if (!sent_to[2 * q]) { P.send[kHaloMeans][q].push_back(e); sent_to[2 * q] = 1; }
      }
    }
  }
  std::vector<int> ghosts;
  for (int e = 0; e < ne; ++e)
    if (ghost_kind[e]) {
      ghosts.push_back(e);
      if (ghost_kind[e] & 1) P.recv[kHaloMeans][P.owner[e]].push_back(e);
      if (ghost_kind[e] & 2) P.recv[kHaloFull][P.owner[e]].push_back(e);
    }
  std::sort(ghosts.begin(), ghosts.end(), [&](int a, int b) { return pos[a] < pos[b]; });
  P.local.insert(P.local.end(), ghosts.begin(), ghosts.end());
  for (int k = 0; k < 2; ++k)
    for (auto& v : P.send[k]) std::sort(v.begin(), v.end());
  return P;
}

}  // namespace dgswem

extern "C" int dgswem_part_halo_ids(const dgswem_cuda_setup* s, int part, int nparts, int peer, int kind,
                                    int* send_ids, int* nsend, int* recv_ids, int* nrecv) {
  return dgswem::guarded([&]() {
    if (!s || !nsend || !nrecv) throw dgswem::Failure(DGSWEM_ERR_ARG, "null argument");
    if (kind != dgswem::kHaloMeans && kind != dgswem::kHaloFull) throw dgswem::Failure(DGSWEM_ERR_ARG, "unknown halo kind");
    if (peer < 0 || peer >= nparts) throw dgswem::Failure(DGSWEM_ERR_ARG, "peer out of range");
    const dgswem::PartPlan P = dgswem::make_part_plan(s, part, nparts);
    const auto& snd = P.send[kind][peer];
    const auto& rcv = P.recv[kind][peer];
    *nsend = (int)snd.size();
    *nrecv = (int)rcv.size();
    if (send_ids) std::copy(snd.begin(), snd.end(), send_ids);
    if (recv_ids) std::copy(rcv.begin(), rcv.end(), recv_ids);
  });
}
