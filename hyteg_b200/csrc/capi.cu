// extern "C" entry points (declared in include/hyteg_b200.h). Each call converts C++
// exceptions into an int status and records the message for hg_last_error().
#include <cuda_runtime.h>

#include <cstring>
#include <map>
#include <string>

#include "../../include/hyteg_b200.h"
#include "server.hpp"
#include "solvers.hpp"
#include "storage.hpp"

struct hg_mesh {
  hg::Discretization* d;
  std::map<std::pair<int, int>, hg::LevelStencils> stencils;  // (level, form)
};

#define HG_TRY try {
#define HG_CATCH                                    \
  }                                                 \
  catch (const hg::Error& e) {                      \
    hg::g_lastError = e.what();                     \
    return e.code;                                  \
  }                                                 \
  catch (const std::exception& e) {                 \
    hg::g_lastError = e.what();                     \
    return HG_ERR_INTERNAL;                         \
  }                                                 \
  return HG_OK;

static hg::Storage& S(hg_storage* h) {
  hg::argCheck(h != nullptr && h->s != nullptr, "null storage handle");
  return *h->s;
}
static const hg::Storage& S(const hg_storage* h) {
  hg::argCheck(h != nullptr && h->s != nullptr, "null storage handle");
  return *h->s;
}
static void levelCheck(const hg::Storage& s, int L) { hg::argCheck(L >= 0 && L <= s.maxLevel(), "level out of range"); }

extern "C" {

const char* hg_last_error(void) { return hg::g_lastError.c_str(); }

int hg_device_count(void) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) {
    (void)cudaGetLastError();
    return 0;
  }
  return n;
}

static int createFrom(const hg::Topology& topo, int maxLevel, hg_storage** out, bool geometryFlags = true) {
  hg::argCheck(out != nullptr, "null output pointer");
  if (hg_device_count() == 0) throw hg::Error(HG_ERR_CUDA, "no CUDA device visible");
  hg::Topology t = topo;
  if (geometryFlags) t.setBoundaryFlags(1, 0);
  hg_storage* h = new hg_storage();
  try {
    h->s = new hg::Storage(t, maxLevel);
  } catch (...) {
    delete h;
    throw;
  }
  *out = h;
  return HG_OK;
}

int hg_storage_create_cuboid(const double lo[3], const double hi[3], int nx, int ny, int nz, int max_level,
                             hg_storage** out) {
  HG_TRY
  hg::argCheck(lo && hi, "null corner");
  hg::argCheck(nx > 0 && ny > 0 && nz > 0, "subdivisions must be positive");
  hg::argCheck(max_level >= 0 && max_level <= 10, "max_level out of range [0,10]");
  for (int d = 0; d < 3; ++d) hg::argCheck(lo[d] < hi[d], "lower corner must be below upper corner");
  return createFrom(hg::meshCuboid(lo, hi, nx, ny, nz), max_level, out);
  HG_CATCH
}

int hg_storage_create_tets(int nverts, const double* coords, int ncells, const int* tets, int max_level,
                           hg_storage** out) {
  HG_TRY
  hg::argCheck(nverts > 0 && ncells > 0 && coords && tets, "empty mesh");
  hg::argCheck(max_level >= 0 && max_level <= 10, "max_level out of range [0,10]");
  std::vector<std::array<double, 3>> c(nverts);
  for (int i = 0; i < nverts; ++i) c[i] = {coords[3 * i], coords[3 * i + 1], coords[3 * i + 2]};
  std::vector<std::array<int, 4>> t(ncells);
  for (int i = 0; i < ncells; ++i) {
    for (int k = 0; k < 4; ++k) {
      hg::argCheck(tets[4 * i + k] >= 0 && tets[4 * i + k] < nverts, "tet vertex index out of range");
      t[i][k] = tets[4 * i + k];
    }
  }
  return createFrom(hg::Topology::fromTets(c, t), max_level, out);
  HG_CATCH
}

static std::vector<std::array<int, 3>> cubeList(int ncubes, const int* cubes) {
  hg::argCheck(ncubes > 0 && cubes != nullptr, "no cubes");
  std::vector<std::array<int, 3>> v(ncubes);
  for (int i = 0; i < ncubes; ++i) {
    for (int d = 0; d < 3; ++d) {
      hg::argCheck(cubes[3 * i + d] > -(1 << 20) && cubes[3 * i + d] < (1 << 20), "cube coordinate out of range");
      v[i][d] = cubes[3 * i + d];
    }
  }
  return v;
}

static hg::Topology cubedDomain(int ncubes, const int* cubes, int cubeType) {
  hg::argCheck(cubeType == 0 || cubeType == 1, "cube type must be 0 or 1");
  return hg::meshCubedDomain(cubeList(ncubes, cubes), cubeType);
}

static hg::Topology gmshTopology(const char* path, int flagsFromFile) {
  hg::argCheck(path != nullptr, "null path");
  try {
    return hg::readGmsh(path, flagsFromFile != 0);
  } catch (const std::runtime_error& e) {
    throw hg::Error(HG_ERR_ARG, e.what());
  }
}

int hg_storage_create_cubed_domain(int ncubes, const int* cubes, int cube_type, int max_level, hg_storage** out) {
  HG_TRY
  hg::argCheck(max_level >= 0 && max_level <= 10, "max_level out of range [0,10]");
  return createFrom(cubedDomain(ncubes, cubes, cube_type), max_level, out);
  HG_CATCH
}

int hg_storage_create_gmsh(const char* path, int max_level, int flags_from_file, hg_storage** out) {
  HG_TRY
  hg::argCheck(max_level >= 0 && max_level <= 10, "max_level out of range [0,10]");
  return createFrom(gmshTopology(path, flags_from_file), max_level, out, flags_from_file == 0);
  HG_CATCH
}

int hg_storage_write_gmsh(const hg_storage* h, const char* path) {
  HG_TRY
  hg::argCheck(h != nullptr && path != nullptr, "null argument");
  try {
    hg::writeGmsh(h->s->disc.topo(), path);
  } catch (const std::runtime_error& e) {
    throw hg::Error(HG_ERR_ARG, e.what());
  }
  HG_CATCH
}

int hg_storage_destroy(hg_storage* h) {
  HG_TRY
  if (!h) return HG_OK;
  delete h->s;
  delete h;
  HG_CATCH
}

int hg_storage_counts(const hg_storage* h, int counts[4]) {
  HG_TRY
  const auto& t = S(h).disc.topo();
  counts[0] = (int)t.verts.size();
  counts[1] = (int)t.edges.size();
  counts[2] = (int)t.faces.size();
  counts[3] = (int)t.cells.size();
  HG_CATCH
}

int hg_storage_set_stream(hg_storage* h, void* stream) {
  HG_TRY
  hg::Storage& s = S(h);
  s.stream = stream ? (cudaStream_t)stream : s.ownStream;
  HG_CATCH
}

int hg_storage_synchronize(hg_storage* h) {
  HG_TRY
  hg::cudaCheck(cudaStreamSynchronize(S(h).stream), "synchronize");
  HG_CATCH
}

int hg_storage_set_l2_budget(hg_storage* h, int64_t bytes) {
  HG_TRY
  S(h).setL2Budget(bytes);
  HG_CATCH
}

int hg_storage_launch_count(const hg_storage* h, unsigned long long* count) {
  HG_TRY
  *count = S(h).launches;
  HG_CATCH
}

int hg_storage_set_cell_coefficients(hg_storage* h, const double* k, int ncells) {
  HG_TRY
  hg::Storage& s = S(h);
  auto& cells = const_cast<hg::Topology&>(s.disc.topo()).cells;
  hg::argCheck(k != nullptr && ncells == (int)cells.size(), "one coefficient per macro-cell required");
  for (int i = 0; i < ncells; ++i) {
    hg::argCheck(k[i] > 0.0, "coefficients must be positive");
    cells[i].k = k[i];
  }
  HG_CATCH
}

int hg_storage_set_concurrent_components(hg_storage* h, int on) {
  HG_TRY
  hg::argCheck(on == 0 || on == 1, "concurrent components: on must be 0 or 1");
  S(h).concurrentComponents = on == 1;
  HG_CATCH
}

int hg_storage_set_sor_fused_phases(hg_storage* h, int on) {
  HG_TRY
  hg::argCheck(on == 0 || on == 1, "fused SOR phases: on must be 0 or 1");
  S(h).fusedSorPhases = on;
  ++S(h).generation;
  HG_CATCH
}

int hg_storage_set_sor_schedule(hg_storage* h, int schedule) {
  HG_TRY
  hg::argCheck(schedule >= 0 && schedule <= 3,
               "SOR schedule must be 0 (single pass), 1 (colour passes), 2 (single pass, short tiles) or 3 "
               "(colour passes in the colour-split order)");
  S(h).sorSchedule = schedule;
  ++S(h).generation;
  HG_CATCH
}

int hg_storage_set_sor_schedule_level(hg_storage* h, int level, int precision, int schedule) {
  HG_TRY
  hg::Storage& s = S(h);
  hg::argCheck(level >= 0 && level <= s.maxLevel(), "level out of range");
  hg::argCheck(precision == 8 || precision == 4, "precision must be 8 or 4");
  hg::argCheck(schedule >= -1 && schedule <= 3, "SOR schedule must be -1 (storage default) or 0..3");
  if ((int)s.sorScheduleLevel.size() < 2 * (s.maxLevel() + 1)) s.sorScheduleLevel.assign(2 * (s.maxLevel() + 1), -1);
  s.sorScheduleLevel[2 * level + (precision == 4 ? 1 : 0)] = schedule;
  ++s.generation;
  HG_CATCH
}

int hg_storage_autotune_sor(hg_storage* h, int min_level, int max_level, int precision, int reps, double* ms,
                            int* chosen) {
  HG_TRY
  hg::Storage& s = S(h);
  s.autotuneSor(min_level, max_level, precision, reps, ms);
  if (chosen)
    for (int L = min_level; L <= max_level; ++L) chosen[L - min_level] = s.sorScheduleLevel[2 * L + (precision == 4)];
  HG_CATCH
}

int hg_primitive_vertices(const hg_storage* h, int kind, int prim, int ids[4], double coords[3], int* flag) {
  HG_TRY
  const auto& t = S(h).disc.topo();
  for (int i = 0; i < 4; ++i) ids[i] = -1;
  switch (kind) {
    case HG_VERTEX:
      hg::argCheck(prim >= 0 && prim < (int)t.verts.size(), "bad vertex");
      ids[0] = prim;
      for (int d = 0; d < 3; ++d) coords[d] = t.verts[prim].x[d];
      *flag = t.verts[prim].flag;
      break;
    case HG_EDGE:
      hg::argCheck(prim >= 0 && prim < (int)t.edges.size(), "bad edge");
      for (int i = 0; i < 2; ++i) ids[i] = t.edges[prim].v[i];
      *flag = t.edges[prim].flag;
      break;
    case HG_FACE:
      hg::argCheck(prim >= 0 && prim < (int)t.faces.size(), "bad face");
      for (int i = 0; i < 3; ++i) ids[i] = t.faces[prim].v[i];
      *flag = t.faces[prim].flag;
      break;
    case HG_CELL:
      hg::argCheck(prim >= 0 && prim < (int)t.cells.size(), "bad cell");
      for (int i = 0; i < 4; ++i) ids[i] = t.cells[prim].v[i];
      *flag = t.cells[prim].flag;
      break;
    default:
      hg::argCheck(false, "bad kind");
  }
  HG_CATCH
}

int hg_primitive_neighbours(const hg_storage* h, int kind, int prim, int which, int* ids, int cap, int* count) {
  HG_TRY
  const auto& t = S(h).disc.topo();
  const std::vector<int>* v = nullptr;
  if (kind == HG_VERTEX) {
    hg::argCheck(prim >= 0 && prim < (int)t.verts.size(), "bad vertex");
    v = which == HG_EDGE ? &t.verts[prim].edges : which == HG_FACE ? &t.verts[prim].faces : &t.verts[prim].cells;
  } else if (kind == HG_EDGE) {
    hg::argCheck(prim >= 0 && prim < (int)t.edges.size(), "bad edge");
    v = which == HG_FACE ? &t.edges[prim].faces : &t.edges[prim].cells;
  } else if (kind == HG_FACE) {
    hg::argCheck(prim >= 0 && prim < (int)t.faces.size(), "bad face");
    v = &t.faces[prim].cells;
  } else {
    hg::argCheck(false, "cells have no higher-dimensional neighbours");
  }
  *count = (int)v->size();
  for (int i = 0; i < (int)v->size() && i < cap; ++i) ids[i] = (*v)[i];
  HG_CATCH
}

int hg_primitive_layout(const hg_storage* h, int level, int kind, int prim, int64_t* offset, int64_t* size) {
  HG_TRY
  const hg::Storage& s = S(h);
  levelCheck(s, level);
  hg::argCheck(kind >= 0 && kind <= 3, "bad kind");
  const auto& lay = s.disc.level(level);
  hg::argCheck(prim >= 0 && prim < (int)lay.off[kind].size(), "bad primitive index");
  *offset = lay.off[kind][prim];
  *size = lay.size[kind][prim];
  HG_CATCH
}

int hg_level_size(const hg_storage* h, int level, int64_t* n) {
  HG_TRY
  const hg::Storage& s = S(h);
  levelCheck(s, level);
  *n = s.disc.level(level).total;
  HG_CATCH
}

int hg_function_create(hg_storage* h, int min_level, int max_level, int precision, int* fn) {
  HG_TRY
  hg::argCheck(fn != nullptr, "null output");
  *fn = S(h).createFunction(min_level, max_level, precision);
  HG_CATCH
}

int hg_function_destroy(hg_storage* h, int fn) {
  HG_TRY
  hg::Storage& s = S(h);
  s.fn(fn);
  s.fns.erase(fn);
  HG_CATCH
}

int hg_function_device_ptr(hg_storage* h, int fn, int level, void** ptr) {
  HG_TRY
  *ptr = S(h).data(fn, level);
  HG_CATCH
}

int hg_function_upload(hg_storage* h, int fn, int level, const void* host, int64_t n) {
  HG_TRY
  hg::Storage& s = S(h);
  hg::Function& f = s.fn(fn);
  hg::argCheck(n == s.disc.level(level).total, "upload size must equal the level buffer size");
  hg::cudaCheck(cudaMemcpyAsync(s.data(fn, level), host, (size_t)n * f.prec, cudaMemcpyHostToDevice, s.stream), "upload");
  hg::cudaCheck(cudaStreamSynchronize(s.stream), "upload sync");
  HG_CATCH
}

int hg_function_upload_async(hg_storage* h, int fn, int level, const void* host, int64_t n, void* stream) {
  HG_TRY
  hg::Storage& s = S(h);
  hg::Function& f = s.fn(fn);
  hg::argCheck(n == s.disc.level(level).total, "upload size must equal the level buffer size");
  hg::cudaCheck(cudaMemcpyAsync(s.data(fn, level), host, (size_t)n * f.prec, cudaMemcpyHostToDevice, (cudaStream_t)stream),
                "upload");
  HG_CATCH
}

int hg_function_download(hg_storage* h, int fn, int level, void* host, int64_t n) {
  HG_TRY
  hg::Storage& s = S(h);
  hg::Function& f = s.fn(fn);
  hg::argCheck(n == s.disc.level(level).total, "download size must equal the level buffer size");
  hg::cudaCheck(cudaMemcpyAsync(host, s.data(fn, level), (size_t)n * f.prec, cudaMemcpyDeviceToHost, s.stream), "download");
  hg::cudaCheck(cudaStreamSynchronize(s.stream), "download sync");
  HG_CATCH
}

int hg_function_download_async(hg_storage* h, int fn, int level, void* host, int64_t n, void* stream) {
  HG_TRY
  hg::Storage& s = S(h);
  hg::Function& f = s.fn(fn);
  hg::argCheck(host != nullptr, "null host buffer");
  hg::argCheck(n == s.disc.level(level).total, "download size must equal the level buffer size");
  hg::cudaCheck(cudaMemcpyAsync(host, s.data(fn, level), (size_t)n * f.prec, cudaMemcpyDeviceToHost, (cudaStream_t)stream),
                "download");
  HG_CATCH
}

int hg_owned_count(hg_storage* h, int level, int64_t* n) {
  HG_TRY
  hg::argCheck(n != nullptr, "null output");
  *n = S(h).ownedPack(level).count;
  HG_CATCH
}

int hg_function_upload_owned_async(hg_storage* h, int fn, int level, const void* host, int64_t n, void* stream) {
  HG_TRY
  S(h).uploadOwned(fn, level, host, n, (cudaStream_t)stream);
  HG_CATCH
}

int hg_function_download_owned_async(hg_storage* h, int fn, int level, void* host, int64_t n, void* stream) {
  HG_TRY
  S(h).downloadOwned(fn, level, host, n, (cudaStream_t)stream);
  HG_CATCH
}

int hg_communicate(hg_storage* h, int fn, int level) {
  HG_TRY
  S(h).communicate(fn, level, (1 << hg::G_COUNT) - 1);
  HG_CATCH
}

int hg_interpolate_const(hg_storage* h, int fn, double value, int level, unsigned flag) {
  HG_TRY
  S(h).lincomb(fn, level, flag, 0, nullptr, nullptr, false, value);
  HG_CATCH
}

int hg_interpolate_expr(hg_storage* h, int fn, int level, unsigned flag, int expr, const double params[4]) {
  HG_TRY
  hg::argCheck(params != nullptr, "null parameters");
  S(h).interpolateExpr(fn, level, flag, expr, params);
  HG_CATCH
}

int hg_assign(hg_storage* h, int dst, int level, unsigned flag, int n, const double* scalars, const int* srcs) {
  HG_TRY
  S(h).lincomb(dst, level, flag, n, scalars, srcs, false, 0.0);
  HG_CATCH
}

int hg_add(hg_storage* h, int dst, int level, unsigned flag, int n, const double* scalars, const int* srcs) {
  HG_TRY
  S(h).lincomb(dst, level, flag, n, scalars, srcs, true, 0.0);
  HG_CATCH
}

int hg_copy_cast(hg_storage* h, int dst, int src, int level, unsigned flag, int add) {
  HG_TRY
  S(h).copyCast(dst, src, level, flag, add != 0);
  HG_CATCH
}

int hg_dot(hg_storage* h, int a, int b, int level, unsigned flag, double* out) {
  HG_TRY
  *out = S(h).dot(a, b, level, flag);
  HG_CATCH
}

int hg_operator_create(hg_storage* h, int form, int min_level, int max_level, int* op) {
  HG_TRY
  *op = S(h).createOperator(form, min_level, max_level);
  HG_CATCH
}

int hg_operator_reassemble(hg_storage* h, int op, int on_device) {
  HG_TRY
  hg::Storage& s = S(h);
  s.op(op);
  hg::argCheck(op != s.structureOp, "internal operator");
  s.reassembleOperator(op, on_device != 0);
  HG_CATCH
}

int hg_operator_destroy(hg_storage* h, int op) {
  HG_TRY
  hg::Storage& s = S(h);
  s.op(op);
  hg::argCheck(op != s.structureOp, "internal operator");
  s.ops.erase(op);
  HG_CATCH
}

int hg_apply(hg_storage* h, int op, int src, int dst, int level, unsigned flag, int update) {
  HG_TRY
  hg::argCheck(update == 0 || update == 1, "update must be 0 (Replace) or 1 (Add)");
  S(h).apply(op, src, dst, level, flag, update);
  HG_CATCH
}

int hg_apply_primitives(hg_storage* h, int op, int src, int dst, int level, unsigned flag, int update, int kinds,
                        int refresh) {
  HG_TRY
  hg::argCheck(update == 0 || update == 1, "update must be 0 (Replace) or 1 (Add)");
  hg::argCheck(kinds > 0 && kinds < 16, "kinds must be a non-empty subset of {vertex, edge, face, cell}");
  S(h).apply(op, src, dst, level, flag, update, kinds, refresh != 0);
  HG_CATCH
}

int hg_residual(hg_storage* h, int op, int x, int b, int r, int level, unsigned flag) {
  HG_TRY
  S(h).residual(op, x, b, r, level, flag);
  HG_CATCH
}

int hg_smooth_sor(hg_storage* h, int op, int dst, int rhs, double omega, int level, unsigned flag, int backwards) {
  HG_TRY
  hg::argCheck(omega > 0.0 && omega < 2.0, "relaxation must lie in (0, 2)");
  S(h).smoothSor(op, dst, rhs, omega, level, flag, backwards != 0);
  HG_CATCH
}

int hg_smooth_sor_primitives(hg_storage* h, int op, int dst, int rhs, double omega, int level, unsigned flag,
                             int backwards, int kinds, int refresh) {
  HG_TRY
  hg::argCheck(omega > 0.0 && omega < 2.0, "relaxation must lie in (0, 2)");
  hg::argCheck(kinds > 0 && kinds < 16, "kinds must be a non-empty subset of {vertex, edge, face, cell}");
  S(h).smoothSor(op, dst, rhs, omega, level, flag, backwards != 0, kinds, refresh != 0);
  HG_CATCH
}

int hg_restrict(hg_storage* h, int fn, int src_level, unsigned flag) {
  HG_TRY
  S(h).restrictFn(fn, src_level, flag);
  HG_CATCH
}

int hg_prolongate(hg_storage* h, int fn, int src_level, unsigned flag, int add) {
  HG_TRY
  S(h).prolongate(fn, src_level, flag, add != 0);
  HG_CATCH
}

int hg_cg_solve(hg_storage* h, int op, int x, int b, int level, int max_iter, double tol, int* iterations,
                double* final_residual) {
  HG_TRY
  hg::Storage& s = S(h);
  const int prec = s.fn(x).prec;
  const int p = s.createFunction(level, level, prec), z = s.createFunction(level, level, prec),
            ap = s.createFunction(level, level, prec), r = s.createFunction(level, level, prec);
  int it = 0;
  double res = 0;
  try {
    it = hg::cgSolve(s, op, x, b, level, max_iter, tol, p, z, ap, r, &res);
  } catch (...) {
    for (int id : {p, z, ap, r}) s.fns.erase(id);
    throw;
  }
  for (int id : {p, z, ap, r}) s.fns.erase(id);
  if (iterations) *iterations = it;
  if (final_residual) *final_residual = res;
  HG_CATCH
}

int hg_gmg_create(hg_storage* h, int op, int min_level, int max_level, int pre_smooth, int post_smooth, double omega,
                  int cycle_type, int coarse_max_iter, double coarse_tol, int precision, int* gmg) {
  HG_TRY
  hg::Storage& s = S(h);
  s.op(op);
  hg::argCheck(min_level >= 0 && max_level <= s.maxLevel() && min_level <= max_level, "invalid level range");
  hg::argCheck(pre_smooth >= 0 && post_smooth >= 0, "negative smoothing steps");
  hg::argCheck(cycle_type == 0 || cycle_type == 1, "cycle type must be 0 (V) or 1 (W)");
  hg::argCheck(omega > 0.0 && omega < 2.0, "relaxation must lie in (0, 2)");
  std::unique_ptr<hg::Gmg> g(new hg::Gmg(s, op, min_level, max_level, pre_smooth, post_smooth, omega, cycle_type,
                                         coarse_max_iter, coarse_tol, precision));
  const int id = s.nextId++;
  s.gmgs[id] = std::move(g);
  *gmg = id;
  HG_CATCH
}

int hg_gmg_destroy(hg_storage* h, int gmg) {
  HG_TRY
  hg::Storage& s = S(h);
  hg::argCheck(s.gmgs.count(gmg) == 1, "unknown multigrid handle");
  s.gmgs.erase(gmg);
  HG_CATCH
}

int hg_gmg_solve(hg_storage* h, int gmg, int x, int b, int level) {
  HG_TRY
  hg::Storage& s = S(h);
  auto it = s.gmgs.find(gmg);
  hg::argCheck(it != s.gmgs.end(), "unknown multigrid handle");
  it->second->solve(x, b, level);
  HG_CATCH
}

// ---------------------------------------------------------------------------------------
// host-only mesh view
// ---------------------------------------------------------------------------------------
static hg_mesh* M(const hg_mesh* m) {
  hg::argCheck(m != nullptr && m->d != nullptr, "null mesh handle");
  return const_cast<hg_mesh*>(m);
}
static const hg::LevelStencils& meshStencil(const hg_mesh* mc, int level, int form) {
  hg_mesh* m = const_cast<hg_mesh*>(mc);
  hg::argCheck(level >= 0 && level <= m->d->maxLevel(), "level out of range");
  hg::argCheck(form == 0 || form == 1, "unknown form");
  auto key = std::make_pair(level, form);
  auto it = m->stencils.find(key);
  if (it == m->stencils.end()) it = m->stencils.emplace(key, hg::assembleStencils(*m->d, level, (hg::FormKind)form)).first;
  return it->second;
}

static int meshFrom(const hg::Topology& topo, int maxLevel, hg_mesh** out, bool geometryFlags = true) {
  hg::argCheck(out != nullptr, "null output pointer");
  hg::Topology t = topo;
  if (geometryFlags) t.setBoundaryFlags(1, 0);
  hg_mesh* m = new hg_mesh();
  try {
    m->d = new hg::Discretization(t, maxLevel);
  } catch (...) {
    delete m;
    throw;
  }
  *out = m;
  return HG_OK;
}

int hg_mesh_create_cuboid(const double lo[3], const double hi[3], int nx, int ny, int nz, int max_level, hg_mesh** out) {
  HG_TRY
  hg::argCheck(lo && hi, "null corner");
  hg::argCheck(nx > 0 && ny > 0 && nz > 0, "subdivisions must be positive");
  hg::argCheck(max_level >= 0 && max_level <= 10, "max_level out of range [0,10]");
  for (int d = 0; d < 3; ++d) hg::argCheck(lo[d] < hi[d], "lower corner must be below upper corner");
  return meshFrom(hg::meshCuboid(lo, hi, nx, ny, nz), max_level, out);
  HG_CATCH
}

int hg_mesh_create_cuboid_copies(int k, int copies, int max_level, hg_mesh** out) {
  HG_TRY
  hg::argCheck(k >= 1 && k <= 16 && copies >= 1 && copies <= 64, "copies of a cube: k in [1, 16], copies in [1, 64]");
  hg::argCheck(max_level >= 0 && max_level <= 10, "max_level out of range [0,10]");
  return meshFrom(hg::meshCuboidCopies(k, copies), max_level, out);
  HG_CATCH
}

int hg_mesh_create_tets(int nverts, const double* coords, int ncells, const int* tets, int max_level, hg_mesh** out) {
  HG_TRY
  hg::argCheck(nverts > 0 && ncells > 0 && coords && tets, "empty mesh");
  hg::argCheck(max_level >= 0 && max_level <= 10, "max_level out of range [0,10]");
  std::vector<std::array<double, 3>> c(nverts);
  for (int i = 0; i < nverts; ++i) c[i] = {coords[3 * i], coords[3 * i + 1], coords[3 * i + 2]};
  std::vector<std::array<int, 4>> t(ncells);
  for (int i = 0; i < ncells; ++i)
    for (int k = 0; k < 4; ++k) {
      hg::argCheck(tets[4 * i + k] >= 0 && tets[4 * i + k] < nverts, "tet vertex index out of range");
      t[i][k] = tets[4 * i + k];
    }
  return meshFrom(hg::Topology::fromTets(c, t), max_level, out);
  HG_CATCH
}

int hg_mesh_create_cubed_domain(int ncubes, const int* cubes, int cube_type, int max_level, hg_mesh** out) {
  HG_TRY
  hg::argCheck(max_level >= 0 && max_level <= 10, "max_level out of range [0,10]");
  return meshFrom(cubedDomain(ncubes, cubes, cube_type), max_level, out);
  HG_CATCH
}

int hg_mesh_create_gmsh(const char* path, int max_level, int flags_from_file, hg_mesh** out) {
  HG_TRY
  hg::argCheck(max_level >= 0 && max_level <= 10, "max_level out of range [0,10]");
  return meshFrom(gmshTopology(path, flags_from_file), max_level, out, flags_from_file == 0);
  HG_CATCH
}

int hg_mesh_write_gmsh(const hg_mesh* m, const char* path) {
  HG_TRY
  hg::argCheck(m != nullptr && path != nullptr, "null argument");
  try {
    hg::writeGmsh(m->d->topo(), path);
  } catch (const std::runtime_error& e) {
    throw hg::Error(HG_ERR_ARG, e.what());
  }
  HG_CATCH
}

int hg_mesh_destroy(hg_mesh* m) {
  HG_TRY
  if (!m) return HG_OK;
  delete m->d;
  delete m;
  HG_CATCH
}

int hg_mesh_counts(const hg_mesh* m, int counts[4]) {
  HG_TRY
  const auto& t = M(m)->d->topo();
  counts[0] = (int)t.verts.size();
  counts[1] = (int)t.edges.size();
  counts[2] = (int)t.faces.size();
  counts[3] = (int)t.cells.size();
  HG_CATCH
}

int hg_mesh_set_cell_coefficients(hg_mesh* m, const double* k, int ncells) {
  HG_TRY
  auto& cells = const_cast<hg::Topology&>(M(m)->d->topo()).cells;
  hg::argCheck(k != nullptr && ncells == (int)cells.size(), "one coefficient per macro-cell required");
  for (int i = 0; i < ncells; ++i) {
    hg::argCheck(k[i] > 0.0, "coefficients must be positive");
    cells[i].k = k[i];
  }
  m->stencils.clear();
  HG_CATCH
}

int hg_mesh_primitive_vertices(const hg_mesh* m, int kind, int prim, int ids[4], double coords[3], int* flag) {
  HG_TRY
  const auto& t = M(m)->d->topo();
  for (int i = 0; i < 4; ++i) ids[i] = -1;
  switch (kind) {
    case HG_VERTEX:
      hg::argCheck(prim >= 0 && prim < (int)t.verts.size(), "bad vertex");
      ids[0] = prim;
      for (int d = 0; d < 3; ++d) coords[d] = t.verts[prim].x[d];
      *flag = t.verts[prim].flag;
      break;
    case HG_EDGE:
      hg::argCheck(prim >= 0 && prim < (int)t.edges.size(), "bad edge");
      for (int i = 0; i < 2; ++i) ids[i] = t.edges[prim].v[i];
      *flag = t.edges[prim].flag;
      break;
    case HG_FACE:
      hg::argCheck(prim >= 0 && prim < (int)t.faces.size(), "bad face");
      for (int i = 0; i < 3; ++i) ids[i] = t.faces[prim].v[i];
      *flag = t.faces[prim].flag;
      break;
    case HG_CELL:
      hg::argCheck(prim >= 0 && prim < (int)t.cells.size(), "bad cell");
      for (int i = 0; i < 4; ++i) ids[i] = t.cells[prim].v[i];
      *flag = t.cells[prim].flag;
      break;
    default:
      hg::argCheck(false, "bad kind");
  }
  HG_CATCH
}

int hg_mesh_primitive_neighbours(const hg_mesh* m, int kind, int prim, int which, int* ids, int cap, int* count) {
  HG_TRY
  const auto& t = M(m)->d->topo();
  const std::vector<int>* v = nullptr;
  if (kind == HG_VERTEX) {
    hg::argCheck(prim >= 0 && prim < (int)t.verts.size(), "bad vertex");
    v = which == HG_EDGE ? &t.verts[prim].edges : which == HG_FACE ? &t.verts[prim].faces : &t.verts[prim].cells;
  } else if (kind == HG_EDGE) {
    hg::argCheck(prim >= 0 && prim < (int)t.edges.size(), "bad edge");
    v = which == HG_FACE ? &t.edges[prim].faces : &t.edges[prim].cells;
  } else if (kind == HG_FACE) {
    hg::argCheck(prim >= 0 && prim < (int)t.faces.size(), "bad face");
    v = &t.faces[prim].cells;
  } else {
    hg::argCheck(false, "cells have no higher-dimensional neighbours");
  }
  *count = (int)v->size();
  for (int i = 0; i < (int)v->size() && i < cap; ++i) ids[i] = (*v)[i];
  HG_CATCH
}

int hg_mesh_primitive_layout(const hg_mesh* m, int level, int kind, int prim, int64_t* offset, int64_t* size) {
  HG_TRY
  const hg::Discretization& d = *M(m)->d;
  hg::argCheck(level >= 0 && level <= d.maxLevel(), "level out of range");
  hg::argCheck(kind >= 0 && kind <= 3, "bad kind");
  const auto& lay = d.level(level);
  hg::argCheck(prim >= 0 && prim < (int)lay.off[kind].size(), "bad primitive index");
  *offset = lay.off[kind][prim];
  *size = lay.size[kind][prim];
  HG_CATCH
}

int hg_mesh_level_size(const hg_mesh* m, int level, int64_t* n) {
  HG_TRY
  const hg::Discretization& d = *M(m)->d;
  hg::argCheck(level >= 0 && level <= d.maxLevel(), "level out of range");
  *n = d.level(level).total;
  HG_CATCH
}

int hg_mesh_slot_info(const hg_mesh* m, int level, double* xyz, signed char* owned, int64_t n) {
  HG_TRY
  const hg::Discretization& d = *M(m)->d;
  hg::argCheck(level >= 0 && level <= d.maxLevel(), "level out of range");
  const auto& lay = d.level(level);
  hg::argCheck(n == lay.total, "buffer size must equal the level size");
  const auto& topo = d.topo();
  const double N = (double)lay.N;
  for (int64_t i = 0; i < n; ++i) owned[i] = -1;
  for (int64_t i = 0; i < 3 * n; ++i) xyz[i] = 0.0;
  for (int kind = 0; kind < 4; ++kind)
    for (size_t p = 0; p < lay.off[kind].size(); ++p)
      for (int64_t s = 0; s < lay.size[kind][p]; ++s) {
        const hg::Bary b = d.slotBary(level, kind, (int)p, s);
        const int64_t g = lay.off[kind][p] + s;
        for (int k = 0; k < 3; ++k) {
          double v = 0.0;
          for (int i = 0; i < b.n; ++i) v += (double)b.b[i] * topo.verts[b.v[i]].x[k];
          xyz[3 * g + k] = v / N;
        }
        const hg::Slot o = d.owner(level, b);
        owned[g] = (o.kind == kind && o.prim == (int)p && o.local == s) ? 1 : 0;
      }
  HG_CATCH
}

int hg_mesh_owned_slots(const hg_mesh* m, int level, int64_t* slots, int64_t* n) {
  HG_TRY
  const hg::Discretization& d = *M(m)->d;
  hg::argCheck(level >= 0 && level <= d.maxLevel(), "level out of range");
  hg::argCheck(n != nullptr, "null output");
  const std::vector<hg::SlotRun> runs = hg::ownedRuns(d, level);
  int64_t count = 0;
  for (const auto& r : runs) count += r.len;
  if (slots) {
    hg::argCheck(*n == count, "slots must hold the owned count");
    int64_t k = 0;
    for (const auto& r : runs)
      for (int64_t i = 0; i < r.len; ++i) slots[k++] = r.slot + i;
  }
  *n = count;
  HG_CATCH
}

int hg_mesh_halo_table(const hg_mesh* m, int level, int group, int64_t* dst, int64_t* src, int64_t* n) {
  HG_TRY
  const hg::Discretization& d = *M(m)->d;
  hg::argCheck(level >= 0 && level <= d.maxLevel(), "level out of range");
  hg::argCheck(group >= 0 && group < hg::G_COUNT, "bad halo group");
  const auto& lay = d.level(level);
  const int64_t cnt = (int64_t)lay.commDst[group].size();
  if (dst && src) {
    hg::argCheck(*n >= cnt, "output too small");
    std::memcpy(dst, lay.commDst[group].data(), cnt * sizeof(int64_t));
    std::memcpy(src, lay.commSrc[group].data(), cnt * sizeof(int64_t));
  }
  *n = cnt;
  HG_CATCH
}

int hg_split_tables_check(int level, int64_t* points, int64_t* mismatches) {
  HG_TRY
  hg::argCheck(level >= 2 && level <= 10 && points && mismatches, "level in [2, 10] and outputs required");
  const int64_t w = (int64_t(1) << level) + 1, N = w - 1;
  auto tet = [](int64_t a) { return a * (a + 1) * (a + 2) / 6; };
  auto natural = [&](int64_t x, int64_t y, int64_t z) {
    const int64_t W = w - z;
    return tet(w) - tet(W) + y * (W + 1) - y * (y + 1) / 2 + x;
  };
  auto split = [&](int64_t x, int64_t y, int64_t z) {  // the permutation, from the coordinates
    const int m = (int)(w - z - y);
    return natural(0, y, z) + hg::dev::splitSub(m, (int)(x & 3)) + (x >> 2);
  };
  // record order C E W N S NW SE TC TW TS TSE BC BE BN BNW
  static const int off[15][3] = {{0, 0, 0},  {1, 0, 0},  {-1, 0, 0}, {0, 1, 0},   {0, -1, 0},
                                 {-1, 1, 0}, {1, -1, 0}, {0, 0, 1},  {-1, 0, 1},  {0, -1, 1},
                                 {1, -1, 1}, {0, 0, -1}, {1, 0, -1}, {0, 1, -1},  {-1, 1, -1}};
  int64_t total = 0, bad = 0;
  for (int col = 0; col < 4; ++col) {
    std::vector<hg::dev::SplitRow> rows;
    std::vector<unsigned> pts;
    hg::splitTables(w, col, rows, pts);
    size_t k = 0;
    for (int64_t z = 1; z <= N - 3; ++z)
      for (int64_t y = 1; y <= N - 2 - z; ++y)
        for (int64_t x = 1; x + y + z <= N - 1; ++x) {
          if (((x + 2 * y + 3 * z) & 3) != col) continue;
          ++total;
          if (k >= pts.size()) {
            ++bad;
            continue;
          }
          const unsigned e = pts[k++];
          const hg::dev::SplitRow& r = rows[e >> hg::dev::kSplitJBits];
          const int64_t j = e & ((1u << hg::dev::kSplitJBits) - 1);
          bool okp = true;
          for (int t = 0; t < 15; ++t)
            okp = okp && r.i[t] + j == split(x + off[t][0], y + off[t][1], z + off[t][2]);
          bad += okp ? 0 : 1;
        }
    bad += (int64_t)(pts.size() - std::min(pts.size(), k));  // table entries without a point
  }
  *points = total;
  *mismatches = bad;
  HG_CATCH
}

int hg_mesh_assembly_plan_check(const hg_mesh* m, int level, int form, int64_t* targets, int64_t* terms,
                                int64_t* mismatches) {
  HG_TRY
  hg::argCheck(targets && terms && mismatches, "null output");
  const auto& st = meshStencil(M(m), level, form);
  const hg::AssemblyPlan p = hg::buildAssemblyPlan(*M(m)->d, level, (hg::FormKind)form);
  const hg::Topology& topo = M(m)->d->topo();
  std::vector<double> ref;  // the assembled values in target order
  for (auto& c : st.cell)
    for (int k = 0; k < 16; ++k) ref.push_back(c[k]);
  for (auto& f : st.face)
    for (int k = 0; k < 16; ++k) ref.push_back(k < (int)f.size() ? f[k].w : 0.0);
  for (auto& e : st.edge)
    for (auto& x : e) ref.push_back(x.w);
  for (auto& v : st.vert)
    for (auto& x : v) ref.push_back(x.w);
  hg::argCheck((int64_t)ref.size() == p.nCell + p.nFace + p.nLow, "plan targets differ from the stencil tables");
  int64_t bad = 0;
  for (int64_t t = 0; t < (int64_t)ref.size(); ++t) {
    const double v = hg::evaluatePlanTarget(p, t, topo);
    if (std::memcmp(&v, &ref[t], sizeof(double)) != 0) ++bad;
  }
  *targets = (int64_t)ref.size();
  *terms = (int64_t)p.terms.size();
  *mismatches = bad;
  HG_CATCH
}

int hg_mesh_cell_stencil(const hg_mesh* m, int level, int form, int cell, double w[15]) {
  HG_TRY
  const auto& st = meshStencil(M(m), level, form);
  hg::argCheck(cell >= 0 && cell < (int)st.cell.size(), "bad cell");
  for (int k = 0; k < 15; ++k) w[k] = st.cell[cell][k];
  HG_CATCH
}

int hg_mesh_face_stencil(const hg_mesh* m, int level, int form, int face, int* layer, int* dx, int* dy, double* w,
                         int cap, int* n) {
  HG_TRY
  const auto& st = meshStencil(M(m), level, form);
  hg::argCheck(face >= 0 && face < (int)st.face.size(), "bad face");
  const auto& e = st.face[face];
  *n = (int)e.size();
  hg::argCheck(cap >= (int)e.size(), "output too small");
  for (size_t k = 0; k < e.size(); ++k) {
    layer[k] = e[k].layer;
    dx[k] = e[k].dx;
    dy[k] = e[k].dy;
    w[k] = e[k].w;
  }
  HG_CATCH
}

int hg_mesh_low_stencil(const hg_mesh* m, int level, int form, int kind, int prim, int64_t* rel, double* w, int cap,
                        int* n) {
  HG_TRY
  const auto& st = meshStencil(M(m), level, form);
  hg::argCheck(kind == HG_EDGE || kind == HG_VERTEX, "kind must be edge or vertex");
  const auto& v = kind == HG_EDGE ? st.edge : st.vert;
  hg::argCheck(prim >= 0 && prim < (int)v.size(), "bad primitive");
  const auto& e = v[prim];
  *n = (int)e.size();
  hg::argCheck(cap >= (int)e.size(), "output too small");
  for (size_t k = 0; k < e.size(); ++k) {
    rel[k] = e[k].rel;
    w[k] = e[k].w;
  }
  HG_CATCH
}

int hg_p2_operator_create(hg_storage* h, int form, int min_level, int max_level, int* op) {
  HG_TRY
  hg::argCheck(op != nullptr, "null output pointer");
  *op = S(h).createP2Operator(form, min_level, max_level);
  HG_CATCH
}

int hg_p2_operator_destroy(hg_storage* h, int op) {
  HG_TRY
  S(h).p2ops.erase(op);
  HG_CATCH
}

int hg_p2_apply(hg_storage* h, int op, int src, int dst, int level, unsigned flag) {
  HG_TRY
  S(h).p2Apply(op, src, dst, -1, level, flag, 0);
  HG_CATCH
}

int hg_p2_residual(hg_storage* h, int op, int x, int b, int r, int level, unsigned flag) {
  HG_TRY
  S(h).p2Apply(op, x, r, b, level, flag, 2);
  HG_CATCH
}

int hg_p2_smooth_sor(hg_storage* h, int op, int x, int b, double omega, int level, unsigned flag, int backwards) {
  HG_TRY
  S(h).p2Sor(op, x, b, omega, level, flag, backwards != 0);
  HG_CATCH
}

int hg_p2_prolongate(hg_storage* h, int fn, int level, unsigned flag, int add) {
  HG_TRY
  S(h).p2Prolongate(fn, level, flag, add != 0);
  HG_CATCH
}

int hg_p2_restrict(hg_storage* h, int fn, int level, unsigned flag) {
  HG_TRY
  S(h).p2Restrict(fn, level, flag);
  HG_CATCH
}

int hg_p2_gmg_create(hg_storage* h, int op, int min_level, int max_level, int pre_smooth, int post_smooth,
                     double omega, int coarse_max_iter, double coarse_tol, int* gmg) {
  HG_TRY
  hg::argCheck(gmg != nullptr && pre_smooth >= 0 && post_smooth >= 0 && coarse_max_iter >= 0, "invalid arguments");
  hg::Storage& s = S(h);
  const int id = s.nextId++;
  s.p2gmgs[id].reset(
      new hg::P2Gmg(s, op, min_level, max_level, pre_smooth, post_smooth, omega, coarse_max_iter, coarse_tol));
  *gmg = id;
  HG_CATCH
}

int hg_p2_gmg_destroy(hg_storage* h, int gmg) {
  HG_TRY
  S(h).p2gmgs.erase(gmg);
  HG_CATCH
}

static hg::P2Gmg& P2G(hg_storage* h, int gmg) {
  auto& m = S(h).p2gmgs;
  auto it = m.find(gmg);
  hg::argCheck(it != m.end(), "unknown P2 multigrid handle");
  return *it->second;
}

int hg_p2_gmg_solve(hg_storage* h, int gmg, int x, int b, int level) {
  HG_TRY
  hg::P2Gmg& g = P2G(h, gmg);
  hg::argCheck(level >= g.minL && level <= g.maxL, "level outside the solver's range");
  g.runCycle(x, b, level);
  HG_CATCH
}

int hg_p2_gmg_solve_to(hg_storage* h, int gmg, int x, int b, int level, double tol, int max_iter, int* iterations,
                       double* rel_residual, double* history, int history_cap) {
  HG_TRY
  hg::argCheck(tol > 0.0 && max_iter >= 0, "tolerance must be positive");
  const int n = P2G(h, gmg).solveTo(x, b, level, tol, max_iter, rel_residual, history, history_cap);
  if (iterations) *iterations = n;
  HG_CATCH
}

int hg_p2p1_stokes_create(hg_storage* h, int min_level, int max_level, int* op) {
  HG_TRY
  hg::argCheck(op != nullptr, "null output pointer");
  *op = S(h).createStokesOperator(min_level, max_level);
  HG_CATCH
}

int hg_p2p1_stokes_apply(hg_storage* h, int op, const int u[3], int p, const int v[3], int q, int level,
                         unsigned flag_velocity, unsigned flag_pressure) {
  HG_TRY
  hg::argCheck(u && v, "null function lists");
  S(h).stokesApply(op, u, p, v, q, level, flag_velocity, flag_pressure);
  HG_CATCH
}

int hg_p2p1_stokes_minres(hg_storage* h, int op, const int u[3], int p, const int f[3], int g, int level, int nu,
                          int max_iter, double tol, int* iterations, double* rel_residual, double* history,
                          int history_cap) {
  HG_TRY
  hg::argCheck(u && f && tol > 0.0 && max_iter >= 0 && nu >= 0, "invalid arguments");
  const int n = hg::stokesMinres(S(h), op, u, p, f, g, level, nu, max_iter, tol, rel_residual, history, history_cap);
  if (iterations) *iterations = n;
  HG_CATCH
}

int hg_p2p1_stokes_uzawa_gmg_create(hg_storage* h, int op, int min_level, int max_level, int pre_smooth,
                                    int post_smooth, double omega, int velocity_sweeps, int* gmg) {
  HG_TRY
  hg::argCheck(gmg != nullptr, "invalid arguments");
  hg::Storage& s = S(h);
  const int id = s.nextId++;
  s.stokesGmgs[id].reset(
      new hg::StokesGmg(s, op, min_level, max_level, pre_smooth, post_smooth, omega, velocity_sweeps));
  *gmg = id;
  HG_CATCH
}

int hg_p2p1_stokes_uzawa_gmg_destroy(hg_storage* h, int gmg) {
  HG_TRY
  S(h).stokesGmgs.erase(gmg);
  HG_CATCH
}

static hg::StokesGmg& SG(hg_storage* h, int gmg) {
  auto& m = S(h).stokesGmgs;
  auto it = m.find(gmg);
  hg::argCheck(it != m.end(), "unknown Stokes multigrid handle");
  return *it->second;
}

int hg_p2p1_stokes_uzawa_smooth(hg_storage* h, int gmg, const int u[3], int p, const int f[3], int g, int level) {
  HG_TRY
  hg::StokesGmg& m = SG(h, gmg);
  hg::argCheck(u && f && level >= m.minL && level <= m.maxL, "invalid arguments");
  m.smooth(u, p, f, g, level);
  HG_CATCH
}

int hg_p2p1_stokes_uzawa_estimate_omega(hg_storage* h, int gmg, int level, int power_iterations, uint64_t seed,
                                        double* omega) {
  HG_TRY
  hg::argCheck(omega != nullptr, "invalid arguments");
  *omega = SG(h, gmg).estimateOmega(level, power_iterations, seed);
  HG_CATCH
}

int hg_p2p1_stokes_uzawa_gmg_solve(hg_storage* h, int gmg, const int u[3], int p, const int f[3], int g, int level) {
  HG_TRY
  hg::StokesGmg& m = SG(h, gmg);
  hg::argCheck(u && f && level >= m.minL && level <= m.maxL, "invalid arguments");
  m.solveRecursively(u, p, f, g, level);
  HG_CATCH
}

int hg_p2p1_stokes_uzawa_gmg_solve_to(hg_storage* h, int gmg, const int u[3], int p, const int f[3], int g, int level,
                                      double tol, int max_iter, int* iterations, double* rel_residual, double* history,
                                      int history_cap) {
  HG_TRY
  hg::argCheck(u && f && tol > 0.0 && max_iter >= 0, "invalid arguments");
  const int n = SG(h, gmg).solveTo(u, p, f, g, level, tol, max_iter, rel_residual, history, history_cap);
  if (iterations) *iterations = n;
  HG_CATCH
}

int hg_p2p1_stokes_minres_mixed(hg_storage* h, int op, const int u[3], int p, const int f[3], int g, int level, int nu,
                                int max_iter, double tol, int precondition_precision, int* iterations,
                                double* rel_residual, double* history, int history_cap) {
  HG_TRY
  hg::argCheck(u && f && tol > 0.0 && max_iter >= 0 && nu >= 0, "invalid arguments");
  const int n = hg::stokesMinres(S(h), op, u, p, f, g, level, nu, max_iter, tol, rel_residual, history, history_cap,
                                 precondition_precision);
  if (iterations) *iterations = n;
  HG_CATCH
}

struct hg_server {
  hg::Server* s;
};

int hg_server_create(int workers, int64_t hbm_budget_bytes, int precision, hg_server** out) {
  HG_TRY
  hg::argCheck(out != nullptr, "null output pointer");
  if (hg_device_count() == 0) throw hg::Error(HG_ERR_CUDA, "no CUDA device visible");
  std::unique_ptr<hg_server> h(new hg_server());
  h->s = new hg::Server(workers, hbm_budget_bytes, precision);
  *out = h.release();
  HG_CATCH
}

int hg_server_destroy(hg_server* srv) {
  HG_TRY
  if (srv) {
    delete srv->s;
    delete srv;
  }
  HG_CATCH
}

static hg::Server& SV(hg_server* h) {
  hg::argCheck(h != nullptr && h->s != nullptr, "null server");
  return *h->s;
}

int hg_server_prewarm(hg_server* srv, int k, int level) {
  HG_TRY
  hg::argCheck(k >= 1 && k <= 16 && level >= 2 && level <= 8, "shape out of range");
  SV(srv).prewarm(k, level);
  HG_CATCH
}

int hg_server_submit(hg_server* srv, int k, int level, double coefficient, uint64_t seed, double tol, int max_iter,
                     int keep_solution, int64_t* id) {
  HG_TRY
  hg::argCheck(id != nullptr, "null id pointer");
  *id = SV(srv).submit(k, level, coefficient, seed, tol, max_iter, keep_solution != 0);
  HG_CATCH
}

int hg_server_wait(hg_server* srv, int64_t id, double timeout_seconds, int* done) {
  HG_TRY
  const bool d = SV(srv).wait(id, timeout_seconds);
  if (done) *done = d ? 1 : 0;
  HG_CATCH
}

int hg_server_result(hg_server* srv, int64_t id, int* status, int* iterations, double* rel_residual, double times[4],
                     int64_t* inner_dofs) {
  HG_TRY
  auto r = SV(srv).request(id);
  if (status) *status = r->status;
  if (iterations) *iterations = r->iterations;
  if (rel_residual) *rel_residual = r->relResidual;
  if (times) {
    times[0] = r->tSubmit;
    times[1] = r->tStart;
    times[2] = r->tSolve;
    times[3] = r->tEnd;
  }
  if (inner_dofs) *inner_dofs = r->innerDofs;
  if (r->status < 0) throw hg::Error(HG_ERR_STATE, "request failed: " + r->error);
  HG_CATCH
}

int hg_server_set_batching(hg_server* srv, int max_level) {
  HG_TRY
  hg::argCheck(max_level >= -1 && max_level <= 8, "batching: max_level must be in [-1, 8]");
  SV(srv).setBatching(max_level);
  HG_CATCH
}

int hg_server_prewarm_batch(hg_server* srv, int k, int level, int copies) {
  HG_TRY
  hg::argCheck(k >= 1 && k <= 16 && level >= 2 && level <= 8, "shape out of range");
  SV(srv).prewarmBatch(k, level, copies);
  HG_CATCH
}

int hg_server_request_batch(hg_server* srv, int64_t id, int* batch_size) {
  HG_TRY
  hg::argCheck(batch_size != nullptr, "null output pointer");
  *batch_size = SV(srv).request(id)->batchSize;
  HG_CATCH
}

int hg_server_request_setup(hg_server* srv, int64_t id, int* built_hierarchy) {
  HG_TRY
  hg::argCheck(built_hierarchy != nullptr, "null output pointer");
  auto r = SV(srv).request(id);
  *built_hierarchy = r->builtHierarchy ? 1 : 0;
  HG_CATCH
}

int hg_server_solution(hg_server* srv, int64_t id, double* host, int64_t n, int64_t* size) {
  HG_TRY
  auto r = SV(srv).request(id);
  hg::argCheck(r->status == 2, "request has not completed");
  hg::argCheck(r->keepSolution, "request was submitted without keep_solution");
  if (size) *size = (int64_t)r->solution.size();
  if (host) {
    hg::argCheck(n >= (int64_t)r->solution.size(), "host buffer too small");
    std::copy(r->solution.begin(), r->solution.end(), host);
  }
  HG_CATCH
}

int hg_server_stats(hg_server* srv, int64_t stats[6]) {
  HG_TRY
  hg::argCheck(stats != nullptr, "null stats");
  SV(srv).stats(stats);
  HG_CATCH
}

int hg_function_fill_random(hg_storage* h, int fn, int level, unsigned flag, uint64_t seed, double lo, double hi) {
  HG_TRY
  hg::argCheck(lo <= hi, "lo must not exceed hi");
  S(h).fillRandom(fn, level, flag, seed, lo, hi);
  HG_CATCH
}

int hg_p2_gmg_set_graphs(hg_storage* h, int gmg, int enable) {
  HG_TRY
  hg::P2Gmg& g = P2G(h, gmg);
  g.graphs = enable != 0;
  if (!g.graphs) g.cache.clear();
  HG_CATCH
}

int hg_gmg_set_graphs(hg_storage* h, int gmg, int enable) {
  HG_TRY
  hg::Storage& s = S(h);
  auto it = s.gmgs.find(gmg);
  hg::argCheck(it != s.gmgs.end(), "unknown multigrid handle");
  it->second->setGraphs(enable != 0);
  HG_CATCH
}

int hg_gmg_set_compact(hg_storage* h, int gmg, int max_dofs, int cluster_blocks) {
  HG_TRY
  hg::Storage& s = S(h);
  auto it = s.gmgs.find(gmg);
  hg::argCheck(it != s.gmgs.end(), "unknown multigrid handle");
  it->second->setCompact(max_dofs, cluster_blocks);
  HG_CATCH
}

int hg_gmg_compact_top(hg_storage* h, int gmg, int* top) {
  HG_TRY
  hg::Storage& s = S(h);
  auto it = s.gmgs.find(gmg);
  hg::argCheck(it != s.gmgs.end(), "unknown multigrid handle");
  hg::argCheck(top != nullptr, "hg_gmg_compact_top: null output");
  *top = it->second->compactTop;
  HG_CATCH
}

int hg_gmg_set_timing(hg_storage* h, int gmg, int enable) {
  HG_TRY
  hg::Storage& s = S(h);
  auto it = s.gmgs.find(gmg);
  hg::argCheck(it != s.gmgs.end(), "unknown multigrid handle");
  it->second->setTiming(enable != 0);
  HG_CATCH
}

int hg_gmg_timing_json(hg_storage* h, int gmg, char* buf, int64_t cap, int64_t* len) {
  HG_TRY
  hg::Storage& s = S(h);
  auto it = s.gmgs.find(gmg);
  hg::argCheck(it != s.gmgs.end(), "unknown multigrid handle");
  hg::argCheck(it->second->timing != nullptr, "timing is off for this solver (hg_gmg_set_timing)");
  hg::argCheck(len != nullptr, "null length");
  const std::string j = it->second->timing->json();
  *len = (int64_t)j.size();
  if (buf && cap > 0) {
    const int64_t n = std::min<int64_t>(cap - 1, (int64_t)j.size());
    std::memcpy(buf, j.data(), (size_t)n);
    buf[n] = 0;
  }
  HG_CATCH
}

int hg_gmg_solve_to(hg_storage* h, int gmg, int x, int b, int level, double tol, int max_iter, int* iterations,
                    double* rel_residual, double* history, int history_cap) {
  HG_TRY
  hg::Storage& s = S(h);
  auto it = s.gmgs.find(gmg);
  hg::argCheck(it != s.gmgs.end(), "unknown multigrid handle");
  hg::argCheck(tol > 0.0 && max_iter >= 0, "tolerance must be positive");
  const int n = it->second->solveTo(x, b, level, tol, max_iter, rel_residual, history, history_cap);
  if (iterations) *iterations = n;
  HG_CATCH
}

}  // extern "C"
