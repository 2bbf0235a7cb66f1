/*
 * Deterministic stand-in for the METIS 4.0.3 / ParMETIS entry points the
 * reference ParGeMSLR calls (prototypes: ParGeMSLR SRC/utils/protos.hpp:283-288,
 * 64-bit idx_t and real_t per metis.patch:1-8).  Test infrastructure for the
 * oracle build only.
 *
 * METIS itself is a third-party dependency that the reference downloads at
 * build time (build.sh:1-5) and that is absent here, so partitions produced by
 * this stand-in differ from upstream METIS ("parity unpinned" against the
 * authors' published partitions).  What matters for the oracle is that the
 * partition is a valid, balanced, deterministic k-way split of the graph.
 *
 * Method: recursive bisection.  A part is split by a breadth-first sweep that
 * starts at a pseudo-peripheral vertex (the end of repeated BFS eccentricity
 * searches), assigning vertices in BFS order to the first side until its
 * vertex weight reaches the target fraction; disconnected pieces are swept in
 * increasing vertex order.  Nested dissection orders (NodeND) come from the
 * same bisection with the second side's boundary vertices moved to a
 * separator that is numbered last.
 */
#include <algorithm>
#include <cstdint>
#include <vector>

namespace {

typedef long int idx;

struct Graph {
   idx n;
   const idx *xadj;
   const idx *adj;
   const idx *vwgt;
};

/* BFS restricted to vertices with mark[v] == tag; returns the visit order
 * (component of src first, then remaining components in increasing id). */
void bfs_order(const Graph &g, const std::vector<idx> &verts, std::vector<int> &mark, int tag,
               idx src, std::vector<idx> &order, std::vector<idx> *dist)
{
   order.clear();
   std::vector<int> seen_tag(0);
   size_t head = 0;
   const int visited = -tag - 1;
   auto push = [&](idx v, idx d) {
      mark[v] = visited;
      order.push_back(v);
      if (dist) (*dist)[v] = d;
   };
   push(src, 0);
   size_t next_seed = 0;
   while (order.size() < verts.size())
   {
      if (head == order.size())
      {
         while (mark[verts[next_seed]] != tag) next_seed++;
         push(verts[next_seed], 0);
      }
      idx v = order[head++];
      idx dv = dist ? (*dist)[v] : 0;
      for (idx e = g.xadj[v]; e < g.xadj[v + 1]; e++)
      {
         idx u = g.adj[e];
         if (u >= 0 && u < g.n && mark[u] == tag) push(u, dv + 1);
      }
   }
   for (idx v : verts) mark[v] = tag;
}

idx pseudo_peripheral(const Graph &g, const std::vector<idx> &verts, std::vector<int> &mark, int tag)
{
   std::vector<idx> order, dist(g.n, 0);
   idx start = verts[0];
   idx best_ecc = -1;
   for (int it = 0; it < 4; it++)
   {
      bfs_order(g, verts, mark, tag, start, order, &dist);
      /* farthest vertex within the start's component */
      idx far = start, ecc = 0;
      for (idx v : order)
      {
         if (dist[v] > ecc) { ecc = dist[v]; far = v; }
         if (v != start && dist[v] == 0) break; /* next component begins */
      }
      if (ecc <= best_ecc) break;
      best_ecc = ecc;
      start = far;
   }
   return start;
}

/* split verts into two sides with weight fraction frac on side 0 */
void bisect(const Graph &g, const std::vector<idx> &verts, std::vector<int> &mark, int tag, double frac,
            std::vector<idx> &side0, std::vector<idx> &side1)
{
   side0.clear();
   side1.clear();
   if (verts.empty()) return;
   idx src = pseudo_peripheral(g, verts, mark, tag);
   std::vector<idx> order;
   bfs_order(g, verts, mark, tag, src, order, nullptr);
   double total = 0.0;
   for (idx v : verts) total += g.vwgt ? (double)g.vwgt[v] : 1.0;
   double target = frac * total, acc = 0.0;
   for (idx v : order)
   {
      double w = g.vwgt ? (double)g.vwgt[v] : 1.0;
      if (acc + 0.5 * w <= target) { side0.push_back(v); acc += w; }
      else side1.push_back(v);
   }
   std::sort(side0.begin(), side0.end());
   std::sort(side1.begin(), side1.end());
}

void recursive_parts(const Graph &g, std::vector<idx> verts, idx nparts, idx first_part,
                     std::vector<int> &mark, int &next_tag, idx *part)
{
   if (nparts <= 1 || verts.size() <= 1)
   {
      for (idx v : verts) part[v] = first_part;
      return;
   }
   idx k0 = nparts / 2, k1 = nparts - k0;
   int tag = next_tag++;
   for (idx v : verts) mark[v] = tag;
   std::vector<idx> s0, s1;
   bisect(g, verts, mark, tag, (double)k0 / (double)nparts, s0, s1);
   for (idx v : verts) mark[v] = 0;
   std::vector<idx>().swap(verts);
   recursive_parts(g, std::move(s0), k0, first_part, mark, next_tag, part);
   recursive_parts(g, std::move(s1), k1, first_part + k0, mark, next_tag, part);
}

idx count_cut(const Graph &g, const idx *part)
{
   idx cut = 0;
   for (idx v = 0; v < g.n; v++)
      for (idx e = g.xadj[v]; e < g.xadj[v + 1]; e++)
         if (part[g.adj[e]] != part[v]) cut++;
   return cut / 2;
}

int partition(idx n, const idx *xadj, const idx *adj, const idx *vwgt, idx nparts, idx *edgecut, idx *part)
{
   Graph g = {n, xadj, adj, vwgt};
   std::vector<idx> verts(n);
   for (idx i = 0; i < n; i++) verts[i] = i;
   std::vector<int> mark(n, 0);
   int next_tag = 1;
   recursive_parts(g, std::move(verts), nparts, 0, mark, next_tag, part);
   if (edgecut) *edgecut = count_cut(g, part);
   return 1; /* METIS_OK */
}

/* nested dissection: order[k] = vertex placed k-th */
void nd_order(const Graph &g, std::vector<idx> verts, std::vector<int> &mark, int &next_tag,
              std::vector<idx> &out)
{
   if (verts.size() <= 16)
   {
      for (idx v : verts) out.push_back(v);
      return;
   }
   int tag = next_tag++;
   for (idx v : verts) mark[v] = tag;
   std::vector<idx> s0, s1, sep, s1_inner;
   bisect(g, verts, mark, tag, 0.5, s0, s1);
   std::vector<char> in0(0);
   for (idx v : s0) mark[v] = -2;
   for (idx v : s1)
   {
      bool boundary = false;
      for (idx e = g.xadj[v]; e < g.xadj[v + 1] && !boundary; e++)
         if (mark[g.adj[e]] == -2) boundary = true;
      (boundary ? sep : s1_inner).push_back(v);
   }
   for (idx v : verts) mark[v] = 0;
   if (s0.empty() || s1_inner.empty())
   {
      for (idx v : verts) out.push_back(v);
      return;
   }
   nd_order(g, std::move(s0), mark, next_tag, out);
   nd_order(g, std::move(s1_inner), mark, next_tag, out);
   for (idx v : sep) out.push_back(v);
}

} // namespace

extern "C" {

int METIS_PartGraphKway(idx *nvtxs, idx *, idx *xadj, idx *adjncy, idx *vwgt, idx *, idx *, idx *nparts,
                        double *, double *, idx *, idx *edgecut, idx *part)
{
   return partition(*nvtxs, xadj, adjncy, vwgt, *nparts, edgecut, part);
}

int METIS_PartGraphRecursive(idx *nvtxs, idx *, idx *xadj, idx *adjncy, idx *vwgt, idx *, idx *, idx *nparts,
                             double *, double *, idx *, idx *edgecut, idx *part)
{
   return partition(*nvtxs, xadj, adjncy, vwgt, *nparts, edgecut, part);
}

int METIS_NodeND(idx *nvtxs, idx *xadj, idx *adjncy, idx *vwgt, idx *, idx *perm, idx *iperm)
{
   idx n = *nvtxs;
   Graph g = {n, xadj, adjncy, vwgt};
   std::vector<idx> verts(n), out;
   for (idx i = 0; i < n; i++) verts[i] = i;
   std::vector<int> mark(n, 0);
   int next_tag = 1;
   out.reserve(n);
   nd_order(g, std::move(verts), mark, next_tag, out);
   /* METIS convention: perm[new] = old is 'iperm' in METIS naming; METIS
    * returns perm[old] = new and iperm[new] = old. */
   for (idx k = 0; k < n; k++)
   {
      iperm[k] = out[k];
      perm[out[k]] = k;
   }
   return 1;
}

/* single-rank ParMETIS: vtxdist = {0, n}, global ids equal local ids */
int ParMETIS_V3_PartKway(idx *vtxdist, idx *xadj, idx *adjncy, idx *vwgt, idx *, idx *, idx *, idx *,
                         idx *nparts, double *, double *, idx *, idx *edgecut, idx *part, int *)
{
   idx n = vtxdist[1] - vtxdist[0];
   return partition(n, xadj, adjncy, vwgt, *nparts, edgecut, part);
}

int ParMETIS_V3_RefineKway(idx *vtxdist, idx *xadj, idx *adjncy, idx *vwgt, idx *, idx *, idx *, idx *,
                           idx *nparts, double *, double *, idx *, idx *edgecut, idx *part, int *)
{
   idx n = vtxdist[1] - vtxdist[0];
   Graph g = {n, xadj, adjncy, vwgt};
   (void)nparts;
   if (edgecut) *edgecut = count_cut(g, part);
   return 1;
}

int ParMETIS_V3_NodeND(idx *vtxdist, idx *xadj, idx *adjncy, idx *, idx *, idx *order, idx *sizes, int *)
{
   idx n = vtxdist[1] - vtxdist[0];
   std::vector<idx> perm(n), iperm(n);
   METIS_NodeND(&n, xadj, adjncy, nullptr, nullptr, perm.data(), iperm.data());
   for (idx i = 0; i < n; i++) order[i] = perm[i];
   sizes[0] = n;
   return 1;
}

} // extern "C"
