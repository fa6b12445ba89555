// gcmf_join_ref_driver.cu -- TEST INFRASTRUCTURE ONLY.  A driver that runs the
// reference's own GCMF join code, built from the reference's sources where they lie
// (oracle/Makefile), to pin the oracle and the engine to the reference's outputs.
// Nothing of the product links or runs it.
//
//   gcmf_join_ref read    <layer.txt> <outdir>            the reference's text reader
//   gcmf_join_ref seqjoin <base.txt> <overlay.txt> <outdir> its CPU MBR join
//   gcmf_join_ref gpujoin <base.txt> <overlay.txt> <outdir> its GPU join stages
//
// Each mode writes one raw little-endian file per array into <outdir> (<name>.bin);
// tests/golden/make_join_goldens.py turns them into fixtures.
//
// Reference functions called (paths relative to the reference repository):
//   ReadTextFormatPolygon2WithVector   SEQ_Overlay.h:285-390
//   IntersectMBR_SEQ                   SEQ_Overlay.h:510-565
//   SortBaseMBROverlap                 Join.h:5-154   (sweep join, GPU_MBR.h:339-539)
//   GetCMBR                            Join.h:397-433 (Get_CMBR, GPU_Join.h:461-508)
//   PointInPolygonTest                 Join.h:437-467 (GPU_Join.h:836-943)
//   CountCMF / ApplyCMF                Join.h:157-294 (GPU_Join.h:511-735)
//   SegmentIntersectJoin               Join.h:356-393 (GPU_Join.h:326-456)
// The stage order and arguments follow spatialJoin3.cu:176-383 with dimSort=1,
// dimSelect=0 (its defaults when no arguments are given).
//
// Inputs must stay inside the reference's fixed limits; tests/golden/make_join_goldens.py
// only generates such layers: coordinates in [1, 999] (16-digit decimal sort keys,
// tokens shorter than 20 characters), at most 64 vertices per polygon (one edge per
// thread of the 128-thread edge-filter blocks: edgeTempList[400], int16 edge ids),
// at most a few thousand polygons per layer (vector[500] per sweep thread, two-level
// prefix sums), and no two MBR coordinates equal to 12 fraction digits.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <sys/stat.h>
#include <cuda_runtime.h>

// GPU_MBR.h:10-11 declare legacy texture references (removed from CUDA 12) that nothing
// uses; this stand-in type lets those two unused declarations compile.
template <class T, int dim = 1, enum cudaTextureReadMode mode = cudaReadModeElementType>
struct texture {};

// the include order of spatialJoin3.cu:1-11
#include "GPU_Manage.h"
#include "Constants.h"
#include "GPU_Test.h"
#include "GPU_MBR.h"
#include "IO.h"
#include "SEQ_Overlay.h"
#include "GPU_Utility.h"
#include "Join.h"

// GH-CUDA/ghcuda.cpp (pulled in by SEQ_Overlay.h) references the GPU clip entry point,
// which lives in another translation unit of the reference; the join modes never reach it.
void calculateIntersections(coord_t*, coord_t*, int, int, coord_t*, int*, long*, int*, long*, int, int, int*,
                            int*, coord_t**, coord_t**, int**, int**, int**, int**, int**, int**, int*) {
  std::fprintf(stderr, "calculateIntersections is not part of this driver\n");
  std::abort();
}

namespace {

std::string g_out;

void dump(const char* name, const void* p, size_t bytes) {
  std::string fn = g_out + "/" + name + ".bin";
  FILE* f = std::fopen(fn.c_str(), "wb");
  if (!f) { std::perror(fn.c_str()); std::exit(2); }
  if (bytes && std::fwrite(p, 1, bytes, f) != bytes) { std::perror(fn.c_str()); std::exit(2); }
  std::fclose(f);
}

template <class T>
void dump_dev(const char* name, const T* d, long n) {
  T* h = (T*)std::malloc(sizeof(T) * (n > 0 ? n : 1));
  if (n > 0 && cudaMemcpy(h, d, sizeof(T) * n, cudaMemcpyDeviceToHost) != cudaSuccess) {
    std::fprintf(stderr, "copy of %s failed\n", name);
    std::exit(3);
  }
  dump(name, h, sizeof(T) * (n > 0 ? n : 0));
  std::free(h);
}

void check(const char* what) {
  cudaError_t e = cudaDeviceSynchronize();
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e != cudaSuccess) {
    std::fprintf(stderr, "%s: %s\n", what, cudaGetErrorString(e));
    std::exit(3);
  }
}

// one layer as the reference's reader leaves it
struct HostLayer {
  long n = 0, nv = 0;
  int* vnum = nullptr;
  long* vps = nullptr;
  mbr_t* key = nullptr;
  coord_t* mbr = nullptr;
  coord_t* xy = nullptr;
};

HostLayer read_layer(const char* path, std::vector<polygon>& gh) {
  struct stat st;
  if (stat(path, &st) != 0) { std::perror(path); std::exit(2); }
  // every vertex and every polygon takes at least two bytes of text: these bounds hold
  // whatever the file's content
  long cap = (long)st.st_size / 2 + 16;
  HostLayer L;
  L.vnum = (int*)std::calloc(cap, sizeof(int));
  L.vps = (long*)std::calloc(cap, sizeof(long));
  L.key = (mbr_t*)std::calloc(4 * cap, sizeof(mbr_t));
  L.mbr = (coord_t*)std::calloc(4 * cap, sizeof(coord_t));
  L.xy = (coord_t*)std::calloc(2 * cap, sizeof(coord_t));
  L.n = ReadTextFormatPolygon2WithVector(path, L.vnum, L.vps, L.key, L.mbr, L.xy, &L.nv, 1, (int)cap, gh);
  return L;
}

void dump_layer(const char* prefix, const HostLayer& L) {
  std::string p(prefix);
  dump((p + "_vnum").c_str(), L.vnum, sizeof(int) * L.n);
  dump((p + "_vps").c_str(), L.vps, sizeof(long) * L.n);
  dump((p + "_key").c_str(), L.key, sizeof(mbr_t) * 4 * L.n);
  dump((p + "_mbr").c_str(), L.mbr, sizeof(coord_t) * 4 * L.n);
  dump((p + "_xy").c_str(), L.xy, sizeof(coord_t) * 2 * L.nv);
}

int mode_seqjoin(const HostLayer& B, const HostLayer& O) {
  int** lists = (int**)std::calloc(B.n + 1, sizeof(int*));
  int* counts = (int*)std::calloc(B.n + 1, sizeof(int));
  IntersectMBR_SEQ(B.n, O.n, B.key, O.key, lists, counts);
  std::vector<int> pb, po;
  for (long i = 0; i < B.n; ++i)
    for (int k = 0; k < counts[i]; ++k) { pb.push_back((int)i); po.push_back(lists[i][k]); }
  dump("seq_b", pb.data(), sizeof(int) * pb.size());
  dump("seq_o", po.data(), sizeof(int) * po.size());
  return 0;
}

int mode_gpujoin(const HostLayer& B, const HostLayer& O) {
  // spatialJoin3.cu:176-195
  int *dbVNum, *doVNum;
  long *dbVPSNum, *doVPSNum;
  coord_t *bCoords, *oCoords;
  mbr_t *dbMBR, *doMBR;
  CopyToGPU((void**)&dbVNum, B.vnum, sizeof(int) * B.n, (char*)"dbVNum", 1);
  CopyToGPU((void**)&doVNum, O.vnum, sizeof(int) * O.n, (char*)"doVNum", 1);
  CopyToGPU((void**)&dbVPSNum, B.vps, sizeof(long) * B.n, (char*)"dbVPSNum", 1);
  CopyToGPU((void**)&doVPSNum, O.vps, sizeof(long) * O.n, (char*)"doVPSNum", 1);
  CopyToGPU((void**)&bCoords, B.xy, sizeof(coord_t) * 2 * B.nv, (char*)"bCoords", 1);
  CopyToGPU((void**)&oCoords, O.xy, sizeof(coord_t) * 2 * O.nv, (char*)"oCoords", 1);
  CopyToGPU((void**)&dbMBR, B.key, 4 * sizeof(mbr_t) * B.n, (char*)"dbMBR", 1);
  CopyToGPU((void**)&doMBR, O.key, 4 * sizeof(mbr_t) * O.n, (char*)"doMBR", 1);
  check("upload");

  // spatialJoin3.cu:226-233: the sweep join
  int *djxyCounter = nullptr, *djxyVector = nullptr;
  long pairNum = SortBaseMBROverlap(B.n, O.n, dbMBR, doMBR, &djxyCounter, &djxyVector, 1, 0);
  check("SortBaseMBROverlap");
  dump_dev("jxy", djxyVector, 2 * pairNum);

  // spatialJoin3.cu:246-253: common MBRs and containment candidates
  int *djxy2IndexList, *djPiPIndexList, *dPiPFlag, *djoinFlag;
  char* dPiPType;
  long eiNum = 0, pipNum = 0, workLoadNum = 0;
  coord_t *dcMBR, *dbMBR2, *doMBR2;
  CopyToGPU((void**)&doMBR2, O.mbr, sizeof(coord_t) * O.n * 4, (char*)"doMBR2", 1);
  CopyToGPU((void**)&dbMBR2, B.mbr, sizeof(coord_t) * B.n * 4, (char*)"dbMBR2", 1);
  GetCMBR(pairNum, djxyVector, dbMBR2, doMBR2, &dcMBR, &djPiPIndexList, &dPiPFlag, &dPiPType, &djoinFlag, &pipNum);
  check("GetCMBR");
  dump_dev("cmbr", dcMBR, 4 * pairNum);
  dump_dev("pip_type", dPiPType, pairNum);
  dump_dev("pip_candidate", dPiPFlag, pairNum);

  // spatialJoin3.cu:262-265: point in polygon
  long wNum = PointInPolygonTest(bCoords, oCoords, pairNum, pipNum, djxyVector, djPiPIndexList, dPiPType, dbVPSNum,
                                 doVPSNum, dPiPFlag, djoinFlag);
  check("PointInPolygonTest");
  dump_dev("pip_flag", dPiPFlag, pairNum);

  // spatialJoin3.cu:288-309: common-MBR edge filter
  poly_size_t *dbEdgeList, *doEdgeList;
  long *dbEdgePSCounter, *doEdgePSCounter, *dWorkLoadPSCounter;
  CountCMF(bCoords, oCoords, pairNum, djxyVector, djoinFlag, dbVNum, doVNum, dbVPSNum, doVPSNum, dcMBR,
           &dbEdgePSCounter, &doEdgePSCounter, &dWorkLoadPSCounter, &djxy2IndexList, &dbEdgeList, &doEdgeList, &eiNum,
           &workLoadNum);
  check("CountCMF");
  ApplyCMF(bCoords, oCoords, pairNum, djxyVector, eiNum, djxy2IndexList, dbVNum, doVNum, dbVPSNum, doVPSNum, dcMBR,
           dbEdgePSCounter, doEdgePSCounter, dbEdgeList, doEdgeList);
  check("ApplyCMF");
  dump_dev("join_flag", djoinFlag, pairNum);
  dump_dev("b_edge_ps", dbEdgePSCounter, pairNum);
  dump_dev("o_edge_ps", doEdgePSCounter, pairNum);
  dump_dev("jxy2", djxy2IndexList, eiNum);
  long nbe = 0, noe = 0;
  if (pairNum > 0) {
    cudaMemcpy(&nbe, dbEdgePSCounter + pairNum - 1, sizeof(long), cudaMemcpyDeviceToHost);
    cudaMemcpy(&noe, doEdgePSCounter + pairNum - 1, sizeof(long), cudaMemcpyDeviceToHost);
  }
  dump_dev("b_edges", dbEdgeList, nbe);
  dump_dev("o_edges", doEdgeList, noe);

  // spatialJoin3.cu:317-318: segment refine
  int* dSegFlag;
  long pairNum3 = SegmentIntersectJoin(bCoords, oCoords, eiNum, djxyVector, djxy2IndexList, dbVPSNum, doVPSNum,
                                       dbEdgePSCounter, doEdgePSCounter, dbEdgeList, doEdgeList, &dSegFlag);
  check("SegmentIntersectJoin");
  dump_dev("seg_flag", dSegFlag, eiNum);
  long counts[6] = {pairNum, pipNum, wNum, eiNum, workLoadNum, pairNum3};
  dump("counts", counts, sizeof(counts));
  return 0;
}

}  // namespace

int main(int argc, char** argv) {
  if (argc < 4) {
    std::fprintf(stderr, "usage: %s read <layer> <outdir> | seqjoin|gpujoin <base> <overlay> <outdir>\n", argv[0]);
    return 1;
  }
  std::string mode = argv[1];
  std::vector<polygon> ghB, ghO;
  if (mode == "read") {
    g_out = argv[3];
    HostLayer L = read_layer(argv[2], ghB);
    dump_layer("layer", L);
    long n[2] = {L.n, L.nv};
    dump("sizes", n, sizeof(n));
    return 0;
  }
  if (argc < 5) return 1;
  g_out = argv[4];
  HostLayer B = read_layer(argv[2], ghB);
  HostLayer O = read_layer(argv[3], ghO);
  if (mode == "seqjoin") return mode_seqjoin(B, O);
  if (mode == "gpujoin") return mode_gpujoin(B, O);
  return 1;
}
