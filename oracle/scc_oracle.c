/*
 * scc_oracle.c — CPU restatement of the reference SCC path.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product (the engine library, the
 * apps, the Python package) links, imports or calls this file.  It is used
 * by tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg, as the
 * checker.
 *
 * Graph layout is the reference's (load.cpp:144-191): vertex ids 1..n,
 * off[n+2] with off[v]..off[v+1] indexing adj[], 1-based neighbour ids.
 * States use the reference bit encoding (scc.h:48-93): B=1 F=2 E=4 T=8 P=16
 * BExt=32 FExt=64.
 *
 * Partition ids follow the engine's exact convention: after a refinement a
 * partition is named by its pivot, the smallest id among its members
 * (the reference names it 3r+k hashed into 2^20 slots, scc_routines.cu:168-176,
 * and elects whichever vertex wins an atomicCAS; both choices only affect
 * which vertex represents a partition, never the final SCCs).
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define ST_B 1u
#define ST_F 2u
#define ST_E 4u
#define ST_T 8u
#define ST_P 16u

/* ------------------------------------------------------------- Tarjan
 * tarjan.cpp:72-240 TR_Decomposition, restated: iterative DFS from vertex 1,
 * then from each next unvisited id (:179-188); popping an unexpanded vertex
 * that was never visited assigns visit/low = time and pushes itself back as
 * expanded followed by ALL successors with from = itself (:117-131); popping
 * an unexpanded visited vertex not yet in a component lowers from's low link
 * to its visit time (:133-137); popping an expanded vertex closes an SCC when
 * visit == low (:141-153, scc_root[member] = the vertex) and then lowers
 * from's low link to its own (:169-173).
 * labels[v] = the component's DFS root (scc_root); returns the count. */
typedef struct {
  uint32_t id; /* bit 31 = expanded */
  uint32_t from;
} tr_item;

long oracle_tarjan(uint32_t n, const uint32_t *off, const uint32_t *adj, uint32_t *labels) {
  if (n == 0) return 0;
  uint32_t *visit = (uint32_t *)calloc((size_t)n + 1, sizeof(uint32_t));
  uint32_t *low = (uint32_t *)calloc((size_t)n + 1, sizeof(uint32_t));
  uint8_t *incomp = (uint8_t *)calloc((size_t)n + 1, 1);
  uint32_t *sccstk = (uint32_t *)malloc(((size_t)n + 1) * sizeof(uint32_t));
  size_t cap = 1024, top = 0, stop = 0;
  tr_item *stk = (tr_item *)malloc(cap * sizeof(tr_item));
  if (!visit || !low || !incomp || !sccstk || !stk) return -1;
  uint32_t time = 1, count = 0, next_seed = 1;
  stk[top++] = (tr_item){1u, 0u};
  for (;;) {
    while (top) {
      tr_item it = stk[--top];
      const uint32_t v = it.id & 0x7fffffffu;
      if (!(it.id & 0x80000000u)) {
        if (visit[v] == 0) {
          visit[v] = low[v] = time++;
          sccstk[stop++] = v;
          const uint32_t deg = off[v + 1] - off[v];
          if (top + 1 + deg > cap) {
            while (top + 1 + deg > cap) cap *= 2;
            stk = (tr_item *)realloc(stk, cap * sizeof(tr_item));
            if (!stk) return -1;
          }
          stk[top++] = (tr_item){v | 0x80000000u, it.from};
          for (uint32_t e = off[v]; e < off[v + 1]; ++e) stk[top++] = (tr_item){adj[e], v};
        } else if (!incomp[v]) {
          if (low[it.from] > visit[v]) low[it.from] = visit[v];
        }
      } else {
        if (visit[v] == low[v] && !incomp[v]) {
          uint32_t w;
          do {
            w = sccstk[--stop];
            labels[w] = v;
            incomp[w] = 1;
          } while (w != v);
          ++count;
        }
        if (!incomp[v] && it.from != 0) {
          if (low[it.from] > low[v]) low[it.from] = low[v];
        }
      }
    }
    while (next_seed <= n && visit[next_seed] != 0) ++next_seed;
    if (next_seed > n) break;
    stk[top++] = (tr_item){next_seed, 0u};
  }
  labels[0] = 0;
  free(visit);
  free(low);
  free(incomp);
  free(sccstk);
  free(stk);
  return (long)count;
}

/* labels -> smallest member id of each class (in place); returns #classes */
long oracle_canonicalize(uint32_t n, uint32_t *labels) {
  uint32_t *mn = (uint32_t *)malloc(((size_t)n + 1) * sizeof(uint32_t));
  if (!mn) return -1;
  for (uint32_t v = 0; v <= n; ++v) mn[v] = 0xffffffffu;
  for (uint32_t v = 1; v <= n; ++v)
    if (labels[v] <= n && v < mn[labels[v]]) mn[labels[v]] = v;
  long cnt = 0;
  for (uint32_t v = 1; v <= n; ++v) {
    labels[v] = mn[labels[v]];
    cnt += labels[v] == v;
  }
  labels[0] = 0;
  free(mn);
  return cnt;
}

/* Independent check that `labels` is THE strongly-connected partition:
 * (1) every class is strongly connected inside itself (forward and backward
 * search from its representative, restricted to the class, reach all
 * members) and (2) the class graph is acyclic (Kahn's algorithm).
 * Returns 0 if valid, 1 if a class is not strongly connected, 2 if the class
 * graph has a cycle, 3 if a label is out of range, -1 on allocation failure. */
int oracle_verify_partition(uint32_t n, const uint32_t *off, const uint32_t *adj, const uint32_t *offT,
                            const uint32_t *adjT, const uint32_t *labels) {
  for (uint32_t v = 1; v <= n; ++v)
    if (labels[v] < 1 || labels[v] > n || labels[labels[v]] != labels[v]) return 3;
  uint32_t *size = (uint32_t *)calloc((size_t)n + 1, sizeof(uint32_t));
  uint8_t *seen = (uint8_t *)calloc((size_t)n + 1, 1);
  uint32_t *q = (uint32_t *)malloc(((size_t)n + 1) * sizeof(uint32_t));
  if (!size || !seen || !q) return -1;
  for (uint32_t v = 1; v <= n; ++v) ++size[labels[v]];
  int rc = 0;
  for (int pass = 0; pass < 2 && rc == 0; ++pass) {
    const uint32_t *o = pass ? offT : off, *a = pass ? adjT : adj;
    memset(seen, 0, (size_t)n + 1);
    for (uint32_t r = 1; r <= n && rc == 0; ++r) {
      if (labels[r] != r) continue;
      size_t h = 0, t = 0;
      q[t++] = r;
      seen[r] = 1;
      while (h < t) {
        const uint32_t v = q[h++];
        for (uint32_t e = o[v]; e < o[v + 1]; ++e) {
          const uint32_t u = a[e];
          if (labels[u] == r && !seen[u]) {
            seen[u] = 1;
            q[t++] = u;
          }
        }
      }
      if (t != size[r]) rc = 1;
    }
  }
  if (rc == 0) {
    /* class DAG check: indegree over inter-class edges (duplicates counted) */
    uint64_t *indeg = (uint64_t *)calloc((size_t)n + 1, sizeof(uint64_t));
    if (!indeg) return -1;
    for (uint32_t v = 1; v <= n; ++v)
      for (uint32_t e = off[v]; e < off[v + 1]; ++e)
        if (labels[adj[e]] != labels[v]) ++indeg[labels[adj[e]]];
    /* members of each class, to walk a class's out-edges */
    uint32_t *start = (uint32_t *)calloc((size_t)n + 2, sizeof(uint32_t));
    uint32_t *mem = (uint32_t *)malloc(((size_t)n + 1) * sizeof(uint32_t));
    if (!start || !mem) return -1;
    for (uint32_t v = 1; v <= n; ++v) ++start[labels[v] + 1];
    for (uint32_t v = 1; v <= n + 1; ++v) start[v] += start[v - 1];
    uint32_t *fill = (uint32_t *)malloc(((size_t)n + 2) * sizeof(uint32_t));
    memcpy(fill, start, ((size_t)n + 2) * sizeof(uint32_t));
    for (uint32_t v = 1; v <= n; ++v) mem[fill[labels[v]]++] = v;
    size_t h = 0, t = 0, ncls = 0;
    for (uint32_t r = 1; r <= n; ++r)
      if (labels[r] == r) {
        ++ncls;
        if (indeg[r] == 0) q[t++] = r;
      }
    while (h < t) {
      const uint32_t r = q[h++];
      for (uint32_t i = start[r]; i < start[r + 1]; ++i) {
        const uint32_t v = mem[i];
        for (uint32_t e = off[v]; e < off[v + 1]; ++e) {
          const uint32_t c = labels[adj[e]];
          if (c != r && --indeg[c] == 0) q[t++] = c;
        }
      }
    }
    if (t != ncls) rc = 2;
    free(indeg);
    free(start);
    free(mem);
    free(fill);
  }
  free(size);
  free(seen);
  free(q);
  return rc;
}

/* ------------------------------------------------------ phase semantics */
static int live_nbr(const uint32_t *off, const uint32_t *adj, uint32_t v, const uint32_t *ranges,
                    const uint8_t *st) {
  for (uint32_t e = off[v]; e < off[v + 1]; ++e) {
    const uint32_t u = adj[e];
    if (u == v || (st[u] & ST_E)) continue;
    if (ranges && ranges[u] != ranges[v]) continue;
    return 1;
  }
  return 0;
}

/* scc_routines.cu:276-394 trim1_kernel / trim_kernel iterated to their
 * fixpoint (trim1 / trim, :582-643): a live vertex without a live
 * (partition-mate, if ranges != NULL) out- or in-neighbour other than itself
 * becomes state 28; labels[v] = v.  The fixpoint does not depend on order.
 * Returns the number of vertices trimmed. */
long oracle_trim(uint32_t n, const uint32_t *off, const uint32_t *adj, const uint32_t *offT, const uint32_t *adjT,
                 const uint32_t *ranges, uint8_t *st, uint32_t *labels) {
  long total = 0;
  int changed = 1;
  while (changed) {
    changed = 0;
    for (uint32_t v = 1; v <= n; ++v) {
      if (st[v] & ST_E) continue;
      if (!live_nbr(off, adj, v, ranges, st) || !live_nbr(offT, adjT, v, ranges, st)) {
        st[v] = 28;
        if (labels) labels[v] = v;
        changed = 1;
        ++total;
      }
    }
  }
  return total;
}

/* reach_q.cu fwd_step/bwd_step (+ the range-free *1 forms) to their
 * fixpoint: every live vertex carrying `bit` (F=2 forward over off/adj, B=1
 * backward over offT/adjT) spreads it to live neighbours in its partition
 * (any partition when ranges == NULL).  Returns the number newly marked. */
long oracle_reach(uint32_t n, const uint32_t *off, const uint32_t *adj, const uint32_t *ranges, uint8_t *st,
                  uint32_t bit) {
  uint32_t *q = (uint32_t *)malloc(((size_t)n + 1) * sizeof(uint32_t));
  if (!q) return -1;
  size_t h = 0, t = 0;
  for (uint32_t v = 1; v <= n; ++v)
    if (!(st[v] & ST_E) && (st[v] & bit)) q[t++] = v;
  long added = 0;
  while (h < t) {
    const uint32_t v = q[h++];
    for (uint32_t e = off[v]; e < off[v + 1]; ++e) {
      const uint32_t u = adj[e];
      if ((st[u] & ST_E) || (st[u] & bit)) continue;
      if (ranges && ranges[u] != ranges[v]) continue;
      st[u] |= (uint8_t)bit;
      q[t++] = u;
      ++added;
    }
  }
  free(q);
  return added;
}

/* scc_routines.cu:187-224 update_kernel: F∩B -> eliminated, label = pivot of
 * its partition (rpivot[range]); every other live vertex moves to partition
 * (range, F, B), state cleared; the smallest id of each non-empty new
 * partition becomes its pivot (state 19) and names it.  rpivot (n+1) maps
 * partition id -> pivot and is updated.  Returns the number of pivots. */
long oracle_update(uint32_t n, uint32_t *ranges, uint8_t *st, uint32_t *labels, uint32_t *rpivot) {
  /* new partition key (range, k) -> smallest member, via sorting-free scan:
   * keys are 3*range+k with range <= n */
  const size_t nk = 3 * ((size_t)n + 1);
  uint32_t *best = (uint32_t *)malloc(nk * sizeof(uint32_t));
  if (!best) return -1;
  for (size_t i = 0; i < nk; ++i) best[i] = 0xffffffffu;
  for (uint32_t v = 1; v <= n; ++v) {
    if (st[v] & ST_E) continue;
    const uint32_t f = (st[v] & ST_F) ? 1u : 0u, b = (st[v] & ST_B) ? 1u : 0u;
    if (f && b) {
      st[v] |= ST_E;
      if (labels) labels[v] = rpivot[ranges[v]];
      continue;
    }
    const size_t key = 3 * (size_t)ranges[v] + f + 2 * b;
    if (v < best[key]) best[key] = v;
  }
  long np = 0;
  for (uint32_t v = 1; v <= n; ++v) {
    if (st[v] & ST_E) continue;
    const uint32_t f = (st[v] & ST_F) ? 1u : 0u, b = (st[v] & ST_B) ? 1u : 0u;
    const size_t key = 3 * (size_t)ranges[v] + f + 2 * b;
    st[v] = 0;
    ranges[v] = best[key];
  }
  for (uint32_t v = 1; v <= n; ++v) {
    if (!(st[v] & ST_E) && ranges[v] == v) {
      st[v] = 19;
      rpivot[v] = v;
      ++np;
    }
  }
  free(best);
  return np;
}

/* scc_routines.cu:397-523 trim2_kernel, evaluated on a snapshot: v whose
 * only live partition-mate out-neighbour (other than itself) u has v as its
 * only one — or the same over in-neighbours — forms the SCC {v, u}: the
 * smaller id gets state 20, the other 4, both labelled with the smaller id.
 * Returns the number of vertices removed. */
static uint32_t single_live(const uint32_t *off, const uint32_t *adj, uint32_t v, const uint32_t *ranges,
                            const uint8_t *st) {
  uint32_t found = 0, cnt = 0;
  for (uint32_t e = off[v]; e < off[v + 1]; ++e) {
    const uint32_t u = adj[e];
    if (u == v || (st[u] & ST_E) || ranges[u] != ranges[v]) continue;
    if (++cnt > 1) return 0;
    found = u;
  }
  return found;
}
static int only_to(const uint32_t *off, const uint32_t *adj, uint32_t u, uint32_t v, const uint32_t *ranges,
                   const uint8_t *st) {
  uint32_t cnt = 0;
  for (uint32_t e = off[u]; e < off[u + 1]; ++e) {
    const uint32_t w = adj[e];
    if (w == u || (st[w] & ST_E) || ranges[w] != ranges[v]) continue;
    if (w != v) return 0;
    ++cnt;
  }
  return cnt == 1;
}
long oracle_trim2(uint32_t n, const uint32_t *off, const uint32_t *adj, const uint32_t *offT, const uint32_t *adjT,
                  const uint32_t *ranges, uint8_t *st, uint32_t *labels) {
  uint32_t *partner = (uint32_t *)calloc((size_t)n + 1, sizeof(uint32_t));
  if (!partner) return -1;
  for (uint32_t v = 1; v <= n; ++v) {
    if (st[v] & ST_E) continue;
    uint32_t u = single_live(off, adj, v, ranges, st);
    if (u && only_to(off, adj, u, v, ranges, st)) {
      partner[v] = u;
      continue;
    }
    u = single_live(offT, adjT, v, ranges, st);
    if (u && only_to(offT, adjT, u, v, ranges, st)) partner[v] = u;
  }
  long cnt = 0;
  for (uint32_t v = 1; v <= n; ++v) {
    if (!partner[v]) continue;
    const uint32_t u = partner[v];
    st[v] = v < u ? 20 : 4;
    if (labels) labels[v] = v < u ? v : u;
    ++cnt;
  }
  free(partner);
  return cnt;
}

/* wcc.cu:7-144 computeWCC + update_ranges2/3, to the fixpoint: colour of a
 * live vertex = smallest id reachable from it through out-edges between live
 * partition-mates; each colour root becomes the pivot (state 19) of a fresh
 * partition named by the root, members take the root's partition.  Pivots
 * of the previous election are expected to be unset (state 0) already.
 * Returns the number of new pivots. */
long oracle_wcc(uint32_t n, const uint32_t *off, const uint32_t *adj, uint32_t *ranges, uint8_t *st,
                uint32_t *rpivot) {
  uint32_t *col = (uint32_t *)malloc(((size_t)n + 1) * sizeof(uint32_t));
  if (!col) return -1;
  for (uint32_t v = 0; v <= n; ++v) col[v] = v;
  int changed = 1;
  while (changed) {
    changed = 0;
    for (uint32_t v = 1; v <= n; ++v) {
      if (st[v] & ST_E) continue;
      uint32_t m = col[v];
      for (uint32_t e = off[v]; e < off[v + 1]; ++e) {
        const uint32_t u = adj[e];
        if ((st[u] & ST_E) || ranges[u] != ranges[v]) continue;
        if (col[u] < m) m = col[u];
      }
      if (col[m] < m) m = col[m];
      if (m < col[v]) {
        col[v] = m;
        changed = 1;
      }
    }
  }
  long np = 0;
  for (uint32_t v = 1; v <= n; ++v) {
    if (st[v] & ST_E) continue;
    ranges[v] = col[v];
    if (col[v] == v) {
      st[v] = 19;
      rpivot[v] = v;
      ++np;
    }
  }
  free(col);
  return np;
}
