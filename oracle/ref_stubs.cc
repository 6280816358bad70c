// TEST INFRASTRUCTURE ONLY (oracle).  Link stubs that let the reference's CPU
// sources link on Linux without OpenCL or METIS.
//
// * OCLwrapper (src/OpenCL/OCLwrapper.h:15-55): every method aborts.  The CPU
//   path (StiffAlgoCPU, ELLmatrix::CG in DEV_CPU/DEV_OMP) never calls it.
// * METIS (un-vendored; only libs/metis/include/metis.h is in the reference):
//   METIS_MeshToDual / METIS_MeshToNodal / METIS_Free are restated from the
//   published METIS 5 semantics for the arguments femColor passes
//   (src/FEM/femColor.cc:103-106, ncommon = 1): two elements are adjacent when
//   they share at least one node.  femColor passes 1-based connectivity with
//   numflag 0; node ids are used as given, with tables sized nn + 1, so the
//   "share a node" relation is exact.  Neighbour order within a row does not
//   affect femColor's first-fit colouring (femColor.cc:146-170), which depends
//   only on the set of neighbour colours.
#include <cstdio>
#include <cstdlib>
#include <vector>
#include <algorithm>
#include "OpenCL/OCLwrapper.h"
#include "metis.h"

static void gf_ocl_unavailable(const char* what) {
  std::fprintf(stderr, "oracle: OpenCL is not available (%s called)\n", what);
  std::abort();
}

OCLwrapper* OCLwrapper::m_oclwrap = nullptr;
OCLwrapper& OCLwrapper::instance() { gf_ocl_unavailable("instance"); return *m_oclwrap; }
OCLwrapper::OCLwrapper() {}
OCLwrapper::~OCLwrapper() {}
void OCLwrapper::setDevice(Device) { gf_ocl_unavailable("setDevice"); }
OCLwrapper::Device OCLwrapper::getDevice() { gf_ocl_unavailable("getDevice"); return NONE; }
void OCLwrapper::setDir(std::string) { gf_ocl_unavailable("setDir"); }
int OCLwrapper::loadSource(std::string) { gf_ocl_unavailable("loadSource"); return 0; }
void OCLwrapper::loadKernel(const char*) { gf_ocl_unavailable("loadKernel"); }
void OCLwrapper::getBuildLog(cl_int, cl_program*, cl_device_id) { gf_ocl_unavailable("getBuildLog"); }
cl_mem OCLwrapper::createBuffer(size_t, cl_mem_flags) { gf_ocl_unavailable("createBuffer"); return nullptr; }
void OCLwrapper::enqueueWriteBuffer(cl_mem, size_t, void*, cl_bool) { gf_ocl_unavailable("enqueueWriteBuffer"); }
void OCLwrapper::enqueueReadBuffer(cl_mem, size_t, void*, cl_bool) { gf_ocl_unavailable("enqueueReadBuffer"); }
void OCLwrapper::setKernelArg(int, size_t, const void*) { gf_ocl_unavailable("setKernelArg"); }
void OCLwrapper::setGlobalWorksize(cl_uint, cl_uint) { gf_ocl_unavailable("setGlobalWorksize"); }
void OCLwrapper::setLocalWorksize(cl_uint, cl_uint) { gf_ocl_unavailable("setLocalWorksize"); }
bool OCLwrapper::localSizeIsOK(size_t) { gf_ocl_unavailable("localSizeIsOK"); return false; }
void OCLwrapper::enquequeNDRangeKernel(cl_uint, bool) { gf_ocl_unavailable("enquequeNDRangeKernel"); }
void OCLwrapper::finish() { gf_ocl_unavailable("finish"); }
void OCLwrapper::releaseMem(cl_mem) { gf_ocl_unavailable("releaseMem"); }
void OCLwrapper::teardown() { gf_ocl_unavailable("teardown"); }
void OCLwrapper::reset() { gf_ocl_unavailable("reset"); }

extern "C" {

int METIS_MeshToDual(idx_t* ne, idx_t* nn, idx_t* eptr, idx_t* eind,
                     idx_t* ncommon, idx_t* numflag, idx_t** r_xadj,
                     idx_t** r_adjncy) {
  (void)numflag;
  const idx_t nelem = *ne;
  const idx_t nnode = *nn;
  const idx_t need = *ncommon < 1 ? 1 : *ncommon;
  // node -> elements incidence, ids used as given (0..nn inclusive)
  std::vector<idx_t> nptr(nnode + 2, 0);
  for (idx_t e = 0; e < nelem; ++e)
    for (idx_t k = eptr[e]; k < eptr[e + 1]; ++k) nptr[eind[k] + 1]++;
  for (idx_t i = 0; i <= nnode; ++i) nptr[i + 1] += nptr[i];
  std::vector<idx_t> nind(nptr[nnode + 1]);
  std::vector<idx_t> fill(nptr.begin(), nptr.end() - 1);
  for (idx_t e = 0; e < nelem; ++e)
    for (idx_t k = eptr[e]; k < eptr[e + 1]; ++k) nind[fill[eind[k]]++] = e;
  std::vector<idx_t> count(nelem, 0);
  std::vector<std::vector<idx_t>> adj(nelem);
  for (idx_t e = 0; e < nelem; ++e) {
    std::vector<idx_t> touched;
    for (idx_t k = eptr[e]; k < eptr[e + 1]; ++k) {
      idx_t node = eind[k];
      for (idx_t q = nptr[node]; q < nptr[node + 1]; ++q) {
        idx_t f = nind[q];
        if (f == e) continue;
        if (count[f]++ == 0) touched.push_back(f);
      }
    }
    for (idx_t f : touched) {
      if (count[f] >= need) adj[e].push_back(f);
      count[f] = 0;
    }
    std::sort(adj[e].begin(), adj[e].end());
  }
  idx_t total = 0;
  for (auto& a : adj) total += (idx_t)a.size();
  idx_t* xadj = (idx_t*)std::malloc(sizeof(idx_t) * (nelem + 1));
  idx_t* adjncy = (idx_t*)std::malloc(sizeof(idx_t) * (total > 0 ? total : 1));
  xadj[0] = 0;
  for (idx_t e = 0; e < nelem; ++e) {
    xadj[e + 1] = xadj[e] + (idx_t)adj[e].size();
    std::copy(adj[e].begin(), adj[e].end(), adjncy + xadj[e]);
  }
  *r_xadj = xadj;
  *r_adjncy = adjncy;
  return METIS_OK;
}

int METIS_MeshToNodal(idx_t* ne, idx_t* nn, idx_t* eptr, idx_t* eind,
                      idx_t* numflag, idx_t** r_xadj, idx_t** r_adjncy) {
  (void)numflag;
  const idx_t nelem = *ne;
  const idx_t nnode = *nn;
  std::vector<std::vector<idx_t>> adj(nnode + 1);
  for (idx_t e = 0; e < nelem; ++e)
    for (idx_t a = eptr[e]; a < eptr[e + 1]; ++a)
      for (idx_t b = eptr[e]; b < eptr[e + 1]; ++b)
        if (eind[a] != eind[b]) adj[eind[a]].push_back(eind[b]);
  idx_t total = 0;
  for (auto& a : adj) {
    std::sort(a.begin(), a.end());
    a.erase(std::unique(a.begin(), a.end()), a.end());
    total += (idx_t)a.size();
  }
  idx_t* xadj = (idx_t*)std::malloc(sizeof(idx_t) * (nnode + 2));
  idx_t* adjncy = (idx_t*)std::malloc(sizeof(idx_t) * (total > 0 ? total : 1));
  xadj[0] = 0;
  for (idx_t i = 0; i <= nnode; ++i) {
    xadj[i + 1] = xadj[i] + (idx_t)adj[i].size();
    std::copy(adj[i].begin(), adj[i].end(), adjncy + xadj[i]);
  }
  *r_xadj = xadj;
  *r_adjncy = adjncy;
  return METIS_OK;
}

int METIS_Free(void* ptr) {
  std::free(ptr);
  return METIS_OK;
}

}  // extern "C"
