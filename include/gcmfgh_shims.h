/*
 * gcmfgh_shims.h -- C++ entry points with the reference's exact signatures, so that the
 * reference's main (main.cpp:15-29) links against libgcmfgh_shims.so unchanged and its
 * two calls reach the B200 engine.  C++ linkage, like the reference (main.h:5-11).
 *
 * spatialJoin  replaces spatialJoin (main.h:5-7, spatialJoin3.cu:40-412).
 *   argv[1] / argv[2] (dimSort, dimSelect, spatialJoin3.cu:50-68) are accepted and have
 *   no effect: the candidate pairs are the same for every sort dimension.  The two input
 *   files, which the reference compiles in through DATASET (spatialJoin3.cu:87-117), are
 *   named by the environment variables GCMFGH_BASE_FILE and GCMFGH_OVERLAY_FILE (GCMF text
 *   format, see gcmfgh_read_text_layer).  Outputs as in the reference: pIDList/qIDList are
 *   host malloc'ed pair lists (caller-owned), *totalPairNum their length, the coordinate
 *   and count pointers are DEVICE pointers in the reference layout that stay valid for the
 *   life of the process.  The pair list is the clip set (containment pairs plus pairs with
 *   intersecting edges), sorted by (base, overlay).  Returns 0, or -1 on an error (the
 *   reference exits instead).
 *
 * ghcuda       replaces ghcuda (main.h:8-11, GH-CUDA/ghcuda.cpp:385-425): clips every
 *   listed pair (swap rule of ghcuda.cpp:64-91) in one batch on the device.  Layers as
 *   spatialJoin returns them (device pointers; other device layers work too, their sizes
 *   then follow from the largest listed id).  The reference writes result polygons only in
 *   debug builds; here they are written in its .poly format (polygon.h:575-584) when the
 *   environment variable GCMFGH_RESULT_FILE names a file.  Returns 0, or -1 on an error.
 *
 * calculateIntersections  replaces the intersection phase of one pair (ghcuda.h:6-14,
 *   gppolyclip_mDIV512.cu:1298-1640), which regularPolygonHandler (ghcuda.cpp:180-340)
 *   calls: P = polygon bPID of the layer at baseCoord, Q = polygon oPID of the layer at
 *   overlayCoords (device layers as spatialJoin returns them; the caller swaps the layers
 *   when Q has more vertices).  Outputs as in the reference, host malloc'ed and freed by the
 *   caller with free(): the merged rings, their (int)(1e7 * alpha) keys, initial labels and
 *   1-based neighbours (see gh_calculate_intersections in gcmfgh.h).  sizeP, sizeQ and cmbr
 *   are not read: the engine takes the ring sizes from the layers and forms the common MBR
 *   from the two polygons' MBRs, as the caller does (ghcuda.cpp:94-125).  *invalid is 1 when
 *   the P-side and Q-side counts differ (arrays NULL, as in the reference) and -1 on an
 *   error (the reference exits instead).
 */
#ifndef GCMFGH_SHIMS_H
#define GCMFGH_SHIMS_H

#ifdef __cplusplus
typedef double coord_t;   /* Types.h:6 */

int spatialJoin(int argc, char* argv[], int** pIDList, int** qIDList, long* totalPairNum,
                coord_t** pBaseCoords, coord_t** pOverlayCoords,
                int** pBVNum, long** pBVPSNum, int** pOVNum, long** pOVPSNum);
int ghcuda(int pIDList[], int qIDList[], int totalNumPairs,
           coord_t* bCoords, coord_t* oCoords,
           int* pBVNum, long* pBVPSNum, int* pOVNum, long* pOVPSNum);
void calculateIntersections(coord_t* baseCoord, coord_t* overlayCoords, int sizeP, int sizeQ, coord_t* cmbr,
                            int* dbVNum, long* dbVPSNum, int* doVNum, long* doVPSNum, int bPID, int oPID,
                            int* countNonDegenIntP, int* countNonDegenIntQ,
                            coord_t** intersectionsP, coord_t** intersectionsQ, int** alphaValuesP,
                            int** alphaValuesQ, int** initLabelsP, int** initLabelsQ,
                            int** neighborP, int** neighborQ, int* invalid);
#endif

#endif /* GCMFGH_SHIMS_H */
