/*
 * RepCut hypergraph restatement (TEST INFRASTRUCTURE ONLY: the checker of
 * the GPU build in jacquard_b200/csrc/repcut.cu; nothing in the product links
 * this file).
 *
 * Follows RCHyperGraph::from_staged_aig (src/repcut.rs:58-176):
 *   - endpoint groups in blocks of 4096 (REPCUT_BITSET_BLOCK_SIZE); per block
 *     the cone of the block's endpoint input pins, found by a traversal that
 *     does not descend through the slice's staged inputs (TopoTraverser,
 *     src/aig.rs:3125-3170);
 *   - the endpoint set of each cone pin is its own endpoints' bits OR the
 *     sets of its fanouts already in the cone, in reverse topological order;
 *   - a cluster is a distinct endpoint set (over all blocks) with at least two
 *     endpoints, counted over pins 1 .. num_pins-1 (the reference's range
 *     excludes the last pin), in first-occurrence order;
 *   - node weights: 1 plus each fanin's weight over its fanout count, in f32
 *     (order of the two fanins as in the reference); endpoint weight = the
 *     f32 sum over its input pins of weight / (number of endpoint inputs on
 *     that pin), rounded as (u64)(sum + 0.5), at least 1.
 * The reference's results depend on its traversal order where a staged
 * input and one of its fanins are both in a cone: the fanin is not
 * descended into from the staged input, so it may come later in the
 * post-order, and then it misses the staged input's set (not yet
 * processed) and the staged input misses its weight.  The traversal is
 * therefore restated exactly (topo below).
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define BLOCK 4096u

static uint32_t g_words; /* words of one full endpoint set */
static const uint64_t *g_sets;

static int cmp_pins(const void *a, const void *b) {
  const uint32_t pa = *(const uint32_t *)a, pb = *(const uint32_t *)b;
  int c = memcmp(g_sets + (size_t)pa * g_words, g_sets + (size_t)pb * g_words, g_words * 8);
  if (c) return c;
  return pa < pb ? -1 : pa > pb;
}

/* TopoTraverser::topo_traverse (src/aig.rs:3125-3170): two-phase iterative
 * DFS, endpoints pushed in order (so the last is explored first), fanin b
 * pushed before a, no descent below staged inputs; returns the post-order. */
static uint32_t topo(uint32_t N, const uint8_t *kind, const uint32_t *fa, const uint32_t *fb,
                     const uint8_t *staged, const uint32_t *start_pins, uint32_t n_start,
                     uint8_t *visited, uint32_t *stack, uint32_t *order) {
  uint32_t sp = 0, n = 0;
  for (uint32_t k = 0; k < n_start; ++k) stack[sp++] = start_pins[k] << 1;  /* Visit */
  while (sp) {
    const uint32_t item = stack[--sp];
    const uint32_t u = item >> 1;
    if (item & 1) {  /* Process */
      order[n++] = u;
      continue;
    }
    if (visited[u]) continue;
    visited[u] = 1;
    stack[sp++] = (u << 1) | 1;
    if (kind[u] == 1 && !staged[u]) {
      if (fb[u] >> 1) stack[sp++] = (fb[u] >> 1) << 1;
      if (fa[u] >> 1) stack[sp++] = (fa[u] >> 1) << 1;
    }
  }
  return n;
}

/* class_of_pin[p] = cluster index (first-occurrence order) or -1;
 * cluster_first[k] / cluster_count[k]; returns the number of clusters, or
 * -1 on allocation failure. */
int jqo_repcut(uint32_t num_pins, const uint8_t *kind, const uint32_t *fa, const uint32_t *fb,
               const uint32_t *fanout_start, const uint32_t *fanouts, const uint8_t *staged,
               uint32_t num_endpoints, const uint32_t *ep_start, const uint32_t *ep_pins,
               int32_t *class_of_pin, uint32_t *cluster_first, uint32_t *cluster_count,
               uint64_t *endpoint_weight) {
  const uint32_t N = num_pins, E = num_endpoints;
  const uint32_t W = (E + 63) / 64 ? (E + 63) / 64 : 1;
  const uint32_t n_ep_pins = E ? ep_start[E] : 0;
  uint64_t *sets = calloc((size_t)(N + 1) * W, 8);
  uint8_t *visited = calloc(N + 1, 1), *done = calloc(N + 1, 1);
  uint32_t *stack = malloc(sizeof(uint32_t) * (2 * (size_t)(N + 1) + n_ep_pins + 8));
  uint32_t *order = malloc(sizeof(uint32_t) * (N + 1));
  if (!sets || !visited || !done || !stack || !order) {
    free(sets); free(visited); free(done); free(stack); free(order);
    return -1;
  }
  for (uint32_t b0 = 0; b0 < E; b0 += BLOCK) {
    const uint32_t b1 = E < b0 + BLOCK ? E : b0 + BLOCK;
    const uint32_t k0 = ep_start[b0], k1 = ep_start[b1];
    memset(visited, 0, N + 1);
    const uint32_t n = topo(N, kind, fa, fb, staged, ep_pins + k0, k1 - k0, visited, stack, order);
    /* own endpoints' bits */
    for (uint32_t e = b0; e < b1; ++e)
      for (uint32_t k = ep_start[e]; k < ep_start[e + 1]; ++k)
        sets[(size_t)ep_pins[k] * W + e / 64] |= 1ull << (e % 64);
    /* reverse post-order: OR the fanouts already processed (vs[j] is Some) */
    memset(done, 0, N + 1);
    const uint32_t w0 = b0 / 64, w1 = (b1 + 63) / 64;
    for (uint32_t oi = n; oi-- > 0;) {
      const uint32_t p = order[oi];
      for (uint32_t k = fanout_start[p]; k < fanout_start[p + 1]; ++k) {
        const uint32_t j = fanouts[k];
        if (!done[j]) continue;
        for (uint32_t w = w0; w < w1; ++w) sets[(size_t)p * W + w] |= sets[(size_t)j * W + w];
      }
      done[p] = 1;
    }
  }
  /* clusters over pins 1 .. N-1 with at least two endpoints */
  uint32_t *pins = malloc(sizeof(uint32_t) * (N + 1));
  uint32_t np = 0;
  for (uint32_t p = 0; p <= N; ++p) class_of_pin[p] = -1;
  for (uint32_t p = 1; p < N; ++p) {
    uint32_t pc = 0;
    for (uint32_t w = 0; w < W; ++w) pc += (uint32_t)__builtin_popcountll(sets[(size_t)p * W + w]);
    if (pc >= 2) pins[np++] = p;
  }
  g_words = W;
  g_sets = sets;
  qsort(pins, np, sizeof(uint32_t), cmp_pins);
  uint32_t ng = 0;
  uint32_t *gfirst = malloc(sizeof(uint32_t) * (np + 1)), *gcount = malloc(sizeof(uint32_t) * (np + 1));
  for (uint32_t i = 0; i < np;) {
    uint32_t j = i;
    while (j < np && memcmp(sets + (size_t)pins[i] * W, sets + (size_t)pins[j] * W, W * 8) == 0) ++j;
    gfirst[ng] = pins[i];  /* sorted by pin within equal sets */
    gcount[ng] = j - i;
    for (uint32_t k = i; k < j; ++k) class_of_pin[pins[k]] = (int32_t)ng;
    ++ng;
    i = j;
  }
  uint32_t *ord = malloc(sizeof(uint32_t) * (ng + 1));
  int32_t *rank = malloc(sizeof(int32_t) * (ng + 1));
  uint32_t n_ord = 0;
  for (uint32_t p = 1; p < N; ++p) {
    const int32_t c = class_of_pin[p];
    if (c >= 0 && gfirst[c] == p) ord[n_ord++] = (uint32_t)c;
  }
  for (uint32_t k = 0; k < n_ord; ++k) {
    rank[ord[k]] = (int32_t)k;
    cluster_first[k] = gfirst[ord[k]];
    cluster_count[k] = gcount[ord[k]];
  }
  for (uint32_t p = 0; p <= N; ++p)
    if (class_of_pin[p] >= 0) class_of_pin[p] = rank[class_of_pin[p]];
  /* node weights in the post-order of a traversal from every endpoint */
  memset(visited, 0, N + 1);
  const uint32_t n_all = topo(N, kind, fa, fb, staged, ep_pins, n_ep_pins, visited, stack, order);
  float *nw = calloc(N + 1, sizeof(float));
  uint32_t *nfe = calloc(N + 1, sizeof(uint32_t));
  for (uint32_t oi = 0; oi < n_all; ++oi) {
    const uint32_t p = order[oi];
    float w = 1.0f;
    if (kind[p] == 1) {
      const uint32_t a = fa[p] >> 1, b = fb[p] >> 1;
      if (a) w += nw[a] / (float)(fanout_start[a + 1] - fanout_start[a]);
      if (b) w += nw[b] / (float)(fanout_start[b + 1] - fanout_start[b]);
    }
    nw[p] = w;
  }
  for (uint32_t k = 0; k < n_ep_pins; ++k) nfe[ep_pins[k]]++;
  for (uint32_t e = 0; e < E; ++e) {
    float tot = 0.0f;
    for (uint32_t k = ep_start[e]; k < ep_start[e + 1]; ++k)
      tot += nw[ep_pins[k]] / (float)nfe[ep_pins[k]];
    const float r = tot + 0.5f;
    uint64_t v = r <= 0.0f ? 0 : (uint64_t)r;
    endpoint_weight[e] = v < 1 ? 1 : v;
  }
  free(nw); free(nfe); free(ord); free(rank); free(gfirst); free(gcount);
  free(pins); free(sets); free(visited); free(done); free(stack); free(order);
  return (int)n_ord;
}
