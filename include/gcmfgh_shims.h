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
#endif

#endif /* GCMFGH_SHIMS_H */
