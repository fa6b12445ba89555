// ghclip_ref_driver.cpp -- TEST INFRASTRUCTURE ONLY (never linked into the product).
//
// Drives the reference's own sequential Greiner-Hormann clipper, compiled from its
// sources where they lie (GH-CUDA/lib/polyclip.h, polygon.h, point2D.h, constants.h),
// so the CPU oracle restatement in oracle/gcmfgh_oracle.cpp can be pinned against the
// reference itself.  Nothing from the reference is copied here; this file only calls
// the reference's functions and data structures.
//
// Two things the reference's CPU path needs that its sources leave out:
//  * Step 1 of labelIntersections (the initial CROSSING/BOUNCING/..._ON classification)
//    is commented out in GH-CUDA/lib/polyclip.h:343-397 because the GPU computes it
//    (GH-CUDA/gppolyclip_mDIV512.cu:1171-1223, which also copies each label to the
//    neighbour on Q at :1219-1220).  initialLabels() below restates that step with the
//    reference's own oracle() (polyclip.h:297) and copies the label to the neighbour,
//    as the GPU path does.
//  * A driver: the reference's main() is commented out (polyclip.h:928-961).
//
// The reference prints progress through `cout` whenever DEBUG_INFO_PRINT is set, which
// GH-CUDA/lib/constants.h hard-wires to 1.  For timing, `cout` is redirected to a stream
// without a buffer, which makes every such print a no-op.
//
// Usage:
//   ghclip_ref text P.poly Q.poly R.poly [union]   (reference .poly text format)
//   ghclip_ref batch in.bin out.bin [union]          (binary pair batch, see readBatch)
//   ghclip_ref time  in.bin reps [union]             (times the batch, prints seconds)
//   ghclip_ref rings in.bin out.bin                  (merged lists + step-1 labels, see below)
//   ghclip_ref mbatch in.bin out.bin [union]         (multi-component pairs, see below)

#include <iostream>
#include <fstream>
#include <cstdlib>
#include <cstdio>
#include <cstdint>
#include <cmath>
#include <string>
#include <vector>
#include <set>
#include <chrono>
#include <bits/stdc++.h>

static std::ostream g_quiet(nullptr);
#define cout g_quiet
#include "polyclip.h"
#undef cout

// Initial classification of every intersection vertex of P, with its label copied to
// the linked vertex of Q (restates polyclip.h:343-397 + gppolyclip_mDIV512.cu:1218-1220).
static IntersectionLabel classifyPair(RelativePositionType qm, RelativePositionType qp) {
  auto has = [&](RelativePositionType a, RelativePositionType b) {
    return (qm == a && qp == b) || (qm == b && qp == a);
  };
  if (has(LEFT, RIGHT)) return CROSSING;
  if ((qm == LEFT && qp == LEFT) || (qm == RIGHT && qp == RIGHT)) return BOUNCING;
  if (has(IS_P_p, RIGHT)) return LEFT_ON;
  if (has(IS_P_p, LEFT)) return RIGHT_ON;
  if (has(IS_P_p, IS_P_m)) return ON_ON;
  if (has(IS_P_m, RIGHT)) return ON_LEFT;
  if (has(IS_P_m, LEFT)) return ON_RIGHT;
  return NONE;
}

static void initialLabels() {
  for (polygon& P : pPolygon)
    for (vertex* I : P.vertices(INTERSECTION)) {
      RelativePositionType qm = oracle(I->neighbour->prev, I->prev, I, I->next);
      RelativePositionType qp = oracle(I->neighbour->next, I->prev, I, I->next);
      IntersectionLabel lab = classifyPair(qm, qp);
      if (lab != NONE) {
        I->label = lab;
        I->neighbour->label = lab;
      }
    }
}

static void runClip() {
  computeIntersections();
  initialLabels();
  labelIntersections();
  createResult();
  cleanUpResult();
}

static void resetGlobals() {
  pPolygon.clear();
  qPolygon.clear();
  resultPolygon.clear();
}

static polygon makePolygon(const double* xy, int n) {
  polygon P;
  for (int i = 0; i < n; ++i) {
    point2D v(xy[2 * i], xy[2 * i + 1]);
    P.newVertex(v, true);
  }
  return P;
}

// Binary batch: int64 npairs; per pair: int32 nP, int32 nQ, f64[2nP], f64[2nQ]
// (open rings, no closing vertex; P is clipped against Q as given).
struct Pair { std::vector<double> p, q; };

static std::vector<Pair> readBatch(const char* fn) {
  std::vector<Pair> out;
  FILE* f = fopen(fn, "rb");
  if (!f) { perror(fn); exit(2); }
  int64_t n = 0;
  if (fread(&n, 8, 1, f) != 1) exit(2);
  out.resize(n);
  for (int64_t k = 0; k < n; ++k) {
    int32_t np, nq;
    if (fread(&np, 4, 1, f) != 1 || fread(&nq, 4, 1, f) != 1) exit(2);
    out[k].p.resize(2 * (size_t)np);
    out[k].q.resize(2 * (size_t)nq);
    if (fread(out[k].p.data(), 8, 2 * (size_t)np, f) != 2 * (size_t)np) exit(2);
    if (fread(out[k].q.data(), 8, 2 * (size_t)nq, f) != 2 * (size_t)nq) exit(2);
  }
  fclose(f);
  return out;
}

int main(int argc, char** argv) {
  if (argc < 4) {
    fprintf(stderr, "usage: %s text P Q R [union] | batch in out [union] | time in reps [union]\n", argv[0]);
    return 2;
  }
  std::string mode = argv[1];
  if (mode == "text") {
    UNION = (argc > 5 && std::string(argv[5]) == "union");
    loadPolygon(pPolygon, std::string(argv[2]));
    loadPolygon(qPolygon, std::string(argv[3]));
    runClip();
    savePolygon(resultPolygon, std::string(argv[4]));
    return 0;
  }
  if (mode == "batch") {
    UNION = (argc > 4 && std::string(argv[4]) == "union");
    std::vector<Pair> pairs = readBatch(argv[2]);
    FILE* f = fopen(argv[3], "wb");
    if (!f) { perror(argv[3]); return 2; }
    int64_t n = (int64_t)pairs.size();
    fwrite(&n, 8, 1, f);
    for (auto& pr : pairs) {
      pPolygon.push_back(makePolygon(pr.p.data(), (int)(pr.p.size() / 2)));
      qPolygon.push_back(makePolygon(pr.q.data(), (int)(pr.q.size() / 2)));
      runClip();
      int32_t nc = 0;
      for (polygon& R : resultPolygon) if (R.root != NULL) ++nc;
      fwrite(&nc, 4, 1, f);
      for (polygon& R : resultPolygon) {
        if (R.root == NULL) continue;
        std::vector<double> xy;
        for (vertex* V : R.vertices(ALL)) { xy.push_back(V->p.x); xy.push_back(V->p.y); }
        int32_t nv = (int32_t)(xy.size() / 2);
        fwrite(&nv, 4, 1, f);
        fwrite(xy.data(), 8, xy.size(), f);
      }
      resetGlobals();
    }
    fclose(f);
    return 0;
  }
  if (mode == "mbatch") {
    // multi-component pairs: int64 npairs; per pair: int32 kP, int32 sizes[kP], int32 kQ,
    // int32 sizes[kQ], then f64 coordinates of P's rings and of Q's rings (open rings).
    // Output as "batch".
    UNION = (argc > 4 && std::string(argv[4]) == "union");
    FILE* fi = fopen(argv[2], "rb");
    FILE* f = fopen(argv[3], "wb");
    if (!fi || !f) { perror("mbatch"); return 2; }
    int64_t n = 0;
    if (fread(&n, 8, 1, fi) != 1) return 2;
    fwrite(&n, 8, 1, f);
    for (int64_t k = 0; k < n; ++k) {
      std::vector<int32_t> sz[2];
      for (int side = 0; side < 2; ++side) {
        int32_t kk = 0;
        if (fread(&kk, 4, 1, fi) != 1) return 2;
        sz[side].resize(kk);
        if (kk > 0 && fread(sz[side].data(), 4, kk, fi) != (size_t)kk) return 2;
      }
      for (int side = 0; side < 2; ++side)
        for (int32_t m : sz[side]) {
          std::vector<double> xy(2 * (size_t)m);
          if (fread(xy.data(), 8, xy.size(), fi) != xy.size()) return 2;
          (side == 0 ? pPolygon : qPolygon).push_back(makePolygon(xy.data(), m));
        }
      runClip();
      int32_t nc = 0;
      for (polygon& R : resultPolygon) if (R.root != NULL) ++nc;
      fwrite(&nc, 4, 1, f);
      for (polygon& R : resultPolygon) {
        if (R.root == NULL) continue;
        std::vector<double> xy;
        for (vertex* V : R.vertices(ALL)) { xy.push_back(V->p.x); xy.push_back(V->p.y); }
        int32_t nv = (int32_t)(xy.size() / 2);
        fwrite(&nv, 4, 1, f);
        fwrite(xy.data(), 8, xy.size(), f);
      }
      resetGlobals();
    }
    fclose(fi);
    fclose(f);
    return 0;
  }
  if (mode == "rings") {
    // The reference's merged lists after computeIntersections and the step-1 labels, for
    // each pair: int32 nP, nQ (list lengths), then per list and vertex in list order from
    // the root: f64 x, y, alpha; int32 source, intersection, label, neighbour position in
    // the other list (-1 = none).
    std::vector<Pair> pairs = readBatch(argv[2]);
    FILE* f = fopen(argv[3], "wb");
    if (!f) { perror(argv[3]); return 2; }
    int64_t n = (int64_t)pairs.size();
    fwrite(&n, 8, 1, f);
    for (auto& pr : pairs) {
      pPolygon.push_back(makePolygon(pr.p.data(), (int)(pr.p.size() / 2)));
      qPolygon.push_back(makePolygon(pr.q.data(), (int)(pr.q.size() / 2)));
      computeIntersections();
      initialLabels();
      std::vector<vertex*> lists[2];
      for (vertex* V : pPolygon[0].vertices(ALL)) lists[0].push_back(V);
      for (vertex* V : qPolygon[0].vertices(ALL)) lists[1].push_back(V);
      int32_t sz[2] = {(int32_t)lists[0].size(), (int32_t)lists[1].size()};
      fwrite(sz, 4, 2, f);
      for (int side = 0; side < 2; ++side) {
        const std::vector<vertex*>& other = lists[1 - side];
        for (vertex* V : lists[side]) {
          double d[3] = {V->p.x, V->p.y, V->alpha};
          int32_t nb = -1;
          for (size_t j = 0; V->neighbour && j < other.size(); ++j)
            if (other[j] == V->neighbour) { nb = (int32_t)j; break; }
          int32_t w[4] = {V->source ? 1 : 0, V->intersection ? 1 : 0, (int32_t)V->label, nb};
          fwrite(d, 8, 3, f);
          fwrite(w, 4, 4, f);
        }
      }
      resetGlobals();
    }
    fclose(f);
    return 0;
  }
  if (mode == "time") {
    UNION = (argc > 4 && std::string(argv[4]) == "union");
    std::vector<Pair> pairs = readBatch(argv[2]);
    int reps = atoi(argv[3]);
    auto t0 = std::chrono::steady_clock::now();
    long long outv = 0;
    for (int r = 0; r < reps; ++r)
      for (auto& pr : pairs) {
        pPolygon.push_back(makePolygon(pr.p.data(), (int)(pr.p.size() / 2)));
        qPolygon.push_back(makePolygon(pr.q.data(), (int)(pr.q.size() / 2)));
        runClip();
        for (polygon& R : resultPolygon)
          if (R.root != NULL) for (vertex* V : R.vertices(ALL)) { (void)V; ++outv; }
        resetGlobals();
      }
    auto t1 = std::chrono::steady_clock::now();
    printf("%.9f %lld\n", std::chrono::duration<double>(t1 - t0).count(), outv);
    return 0;
  }
  return 2;
}
