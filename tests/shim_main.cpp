// The reference's main (main.cpp:15-29), written out against include/gcmfgh_shims.h:
// spatialJoin's outputs go straight into ghcuda, with the pair count narrowed to int.
#include "gcmfgh_shims.h"

int main(int argc, char* argv[]) {
  long totalPairNum;
  int *pIDList, *qIDList;
  coord_t *pBaseCoords, *pOverlayCoords;
  int *pBVNum, *pOVNum;
  long *pBVPSNum, *pOVPSNum;
  if (spatialJoin(argc, argv, &pIDList, &qIDList, &totalPairNum, &pBaseCoords, &pOverlayCoords, &pBVNum,
                  &pBVPSNum, &pOVNum, &pOVPSNum) != 0)
    return 1;
  if (ghcuda(pIDList, qIDList, totalPairNum, pBaseCoords, pOverlayCoords, pBVNum, pBVPSNum, pOVNum, pOVPSNum) != 0)
    return 2;
  return 0;
}
