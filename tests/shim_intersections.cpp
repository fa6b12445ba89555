// The reference's per-pair intersection phase (regularPolygonHandler, ghcuda.cpp:180-226)
// written out against include/gcmfgh_shims.h: spatialJoin's outputs, then
// calculateIntersections on the first argv[3] pairs of the pair list (P = base polygon,
// no swap).  Every pair's outputs go to the binary file argv[4]: int32 n_p, n_q, invalid,
// then (unless invalid) f64 xy_p[2 n_p], xy_q[2 n_q], int32 alpha_p, alpha_q, label_p,
// label_q, neighbor_p, neighbor_q.  The arrays are released with free(), as the reference
// caller does (ghcuda.cpp:325-336).
#include <cstdio>
#include <cstdlib>
#include "gcmfgh_shims.h"

int main(int argc, char* argv[]) {
  if (argc < 5) return 3;
  long totalPairNum;
  int *pIDList, *qIDList;
  coord_t *pBaseCoords, *pOverlayCoords;
  int *pBVNum, *pOVNum;
  long *pBVPSNum, *pOVPSNum;
  if (spatialJoin(argc, argv, &pIDList, &qIDList, &totalPairNum, &pBaseCoords, &pOverlayCoords, &pBVNum,
                  &pBVPSNum, &pOVNum, &pOVPSNum) != 0)
    return 1;
  long n = atol(argv[3]);
  if (n > totalPairNum) n = totalPairNum;
  FILE* f = fopen(argv[4], "wb");
  if (!f) return 4;
  fwrite(&n, sizeof(long), 1, f);
  for (long k = 0; k < n; ++k) {
    int cP = 0, cQ = 0, invalid = 0;
    coord_t *xyP, *xyQ;
    int *aP, *aQ, *lP, *lQ, *nP, *nQ;
    coord_t cmbr[4] = {0, 0, 0, 0};
    calculateIntersections(pBaseCoords, pOverlayCoords, 0, 0, cmbr, pBVNum, pBVPSNum, pOVNum, pOVPSNum,
                           pIDList[k], qIDList[k], &cP, &cQ, &xyP, &xyQ, &aP, &aQ, &lP, &lQ, &nP, &nQ, &invalid);
    if (invalid < 0) return 2;
    int head[3] = {cP, cQ, invalid};
    fwrite(head, sizeof(int), 3, f);
    if (invalid) continue;
    fwrite(xyP, sizeof(coord_t), 2 * (size_t)cP, f);
    fwrite(xyQ, sizeof(coord_t), 2 * (size_t)cQ, f);
    int* arrs[6] = {aP, aQ, lP, lQ, nP, nQ};
    for (int i = 0; i < 6; ++i) {
      fwrite(arrs[i], sizeof(int), (size_t)(i % 2 == 0 ? cP : cQ), f);
      free(arrs[i]);
    }
    free(xyP);
    free(xyQ);
  }
  fclose(f);
  return 0;
}
