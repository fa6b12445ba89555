// shims.cpp -- the reference's C++ entry points (include/gcmfgh_shims.h) over the C ABI.
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <vector>
#include "../../include/gcmfgh.h"
#include "../../include/gcmfgh_shims.h"

namespace {

// Process-wide state of the shims; like the reference, what spatialJoin hands out lives
// until the process ends (it is never freed).
struct ShimState {
  gcmfgh_ctx* ctx = nullptr;
  gcmfgh_text_layer hb{}, ho{};
  gcmfgh_layer db{}, dO{};
  bool loaded = false;
};

ShimState& state() {
  static ShimState* s = new ShimState();
  return *s;
}

bool ensure_ctx() {
  ShimState& S = state();
  if (S.ctx) return true;
  return gcmfgh_create(0, &S.ctx) == GCMFGH_OK;
}

gcmfgh_layer host_view(const gcmfgh_text_layer& t) {
  return gcmfgh_layer{t.coords, t.vnum, t.vps, t.n_polys, t.n_vertices};
}

// polygon.h:575-584: "x y," per vertex on its own line, ';' after the last one, with the
// default ostream precision (6 significant digits)
void write_components(FILE* f, const int32_t* csz, int64_t nc, const double* xy) {
  int64_t v = 0;
  for (int64_t c = 0; c < nc; ++c) {
    for (int32_t k = 0; k < csz[c]; ++k, ++v)
      std::fprintf(f, "%g %g%s", xy[2 * v], xy[2 * v + 1], k + 1 < csz[c] ? ",\n" : ";\n");
  }
}

}  // namespace

int spatialJoin(int argc, char* argv[], int** pIDList, int** qIDList, long* totalPairNum,
                coord_t** pBaseCoords, coord_t** pOverlayCoords,
                int** pBVNum, long** pBVPSNum, int** pOVNum, long** pOVPSNum) {
  (void)argc;
  (void)argv;
  if (!pIDList || !qIDList || !totalPairNum || !pBaseCoords || !pOverlayCoords || !pBVNum || !pBVPSNum ||
      !pOVNum || !pOVPSNum)
    return -1;
  const char* fb = std::getenv("GCMFGH_BASE_FILE");
  const char* fo = std::getenv("GCMFGH_OVERLAY_FILE");
  if (!fb || !fo || !ensure_ctx()) return -1;
  ShimState& S = state();
  gcmfgh_free_text_layer(&S.hb);
  gcmfgh_free_text_layer(&S.ho);
  if (gcmfgh_read_text_layer(fb, 0, &S.hb) != GCMFGH_OK || gcmfgh_read_text_layer(fo, 0, &S.ho) != GCMFGH_OK)
    return -1;
  gcmfgh_layer hb = host_view(S.hb), ho = host_view(S.ho);
  if (gcmfgh_upload_layer(S.ctx, &hb, &S.db) != GCMFGH_OK || gcmfgh_upload_layer(S.ctx, &ho, &S.dO) != GCMFGH_OK)
    return -1;
  S.loaded = true;
  gcmfgh_join_info ji;
  if (gcmf_join(S.ctx, &S.db, &S.dO, &ji) != GCMFGH_OK) return -1;
  const int64_t n = ji.n_clip;
  int* p = static_cast<int*>(std::malloc(sizeof(int) * std::max<int64_t>(n, 1)));
  int* q = static_cast<int*>(std::malloc(sizeof(int) * std::max<int64_t>(n, 1)));
  if (!p || !q) { std::free(p); std::free(q); return -1; }
  int64_t bytes = 0;
  if (n > 0 && (gcmf_join_get(S.ctx, GCMF_CLIP_BASE, p, sizeof(int) * n, 0, &bytes) != GCMFGH_OK ||
                gcmf_join_get(S.ctx, GCMF_CLIP_OVERLAY, q, sizeof(int) * n, 0, &bytes) != GCMFGH_OK)) {
    std::free(p); std::free(q);
    return -1;
  }
  *pIDList = p;
  *qIDList = q;
  *totalPairNum = (long)n;
  *pBaseCoords = const_cast<coord_t*>(S.db.coords);
  *pOverlayCoords = const_cast<coord_t*>(S.dO.coords);
  *pBVNum = const_cast<int*>(S.db.vnum);
  *pBVPSNum = reinterpret_cast<long*>(const_cast<int64_t*>(S.db.vps));
  *pOVNum = const_cast<int*>(S.dO.vnum);
  *pOVPSNum = reinterpret_cast<long*>(const_cast<int64_t*>(S.dO.vps));
  return 0;
}

int ghcuda(int pIDList[], int qIDList[], int totalNumPairs, coord_t* bCoords, coord_t* oCoords,
           int* pBVNum, long* pBVPSNum, int* pOVNum, long* pOVPSNum) {
  if (totalNumPairs < 0 || (totalNumPairs > 0 && (!pIDList || !qIDList)) || !ensure_ctx()) return -1;
  ShimState& S = state();
  gcmfgh_layer b{bCoords, pBVNum, reinterpret_cast<const int64_t*>(pBVPSNum), 0, 0};
  gcmfgh_layer o{oCoords, pOVNum, reinterpret_cast<const int64_t*>(pOVPSNum), 0, 0};
  if (S.loaded && bCoords == S.db.coords && oCoords == S.dO.coords) {
    b = S.db;
    o = S.dO;
  } else {
    int mb = -1, mo = -1;
    for (int k = 0; k < totalNumPairs; ++k) { mb = std::max(mb, pIDList[k]); mo = std::max(mo, qIDList[k]); }
    b.n_polys = mb + 1;
    o.n_polys = mo + 1;
  }
  gcmfgh_clip_info ci;
  if (gh_clip_batch_host_ids(S.ctx, &b, &o, pIDList, qIDList, totalNumPairs, &ci) != GCMFGH_OK) return -1;
  const char* out = std::getenv("GCMFGH_RESULT_FILE");
  if (out) {
    std::vector<int32_t> csz(std::max<int64_t>(ci.n_components, 1));
    std::vector<double> xy(2 * std::max<int64_t>(ci.n_vertices, 1));
    int64_t bytes = 0;
    if (ci.n_components > 0 &&
        (gh_clip_get(S.ctx, GH_COMP_SIZE, csz.data(), sizeof(int32_t) * csz.size(), 0, &bytes) != GCMFGH_OK ||
         gh_clip_get(S.ctx, GH_XY, xy.data(), sizeof(double) * xy.size(), 0, &bytes) != GCMFGH_OK))
      return -1;
    FILE* f = std::fopen(out, "w");
    if (!f) return -1;
    write_components(f, csz.data(), ci.n_components, xy.data());
    std::fclose(f);
  }
  return 0;
}

void calculateIntersections(coord_t* baseCoord, coord_t* overlayCoords, int sizeP, int sizeQ, coord_t* cmbr,
                            int* dbVNum, long* dbVPSNum, int* doVNum, long* doVPSNum, int bPID, int oPID,
                            int* countNonDegenIntP, int* countNonDegenIntQ,
                            coord_t** intersectionsP, coord_t** intersectionsQ, int** alphaValuesP,
                            int** alphaValuesQ, int** initLabelsP, int** initLabelsQ,
                            int** neighborP, int** neighborQ, int* invalid) {
  (void)sizeP;
  (void)sizeQ;
  (void)cmbr;
  int** outs[6] = {alphaValuesP, alphaValuesQ, initLabelsP, initLabelsQ, neighborP, neighborQ};
  for (int** o : outs)
    if (o) *o = nullptr;
  if (intersectionsP) *intersectionsP = nullptr;
  if (intersectionsQ) *intersectionsQ = nullptr;
  if (countNonDegenIntP) *countNonDegenIntP = 0;
  if (countNonDegenIntQ) *countNonDegenIntQ = 0;
  if (!invalid) return;
  *invalid = -1;
  if (!countNonDegenIntP || !countNonDegenIntQ || !intersectionsP || !intersectionsQ || !alphaValuesP ||
      !alphaValuesQ || !initLabelsP || !initLabelsQ || !neighborP || !neighborQ || bPID < 0 || oPID < 0 ||
      !ensure_ctx())
    return;
  ShimState& S = state();
  gcmfgh_layer b{baseCoord, dbVNum, reinterpret_cast<const int64_t*>(dbVPSNum), (int64_t)bPID + 1, 0};
  gcmfgh_layer o{overlayCoords, doVNum, reinterpret_cast<const int64_t*>(doVPSNum), (int64_t)oPID + 1, 0};
  gcmfgh_intersections x;
  if (gh_calculate_intersections(S.ctx, &b, bPID, &o, oPID, &x) != GCMFGH_OK) return;
  *countNonDegenIntP = (int)x.n_p;
  *countNonDegenIntQ = (int)x.n_q;
  *invalid = x.invalid;
  // ownership of the malloc'ed arrays passes to the caller, as in the reference
  *intersectionsP = x.xy_p;
  *intersectionsQ = x.xy_q;
  *alphaValuesP = x.alpha_p;
  *alphaValuesQ = x.alpha_q;
  *initLabelsP = x.label_p;
  *initLabelsQ = x.label_q;
  *neighborP = x.neighbor_p;
  *neighborQ = x.neighbor_q;
}
