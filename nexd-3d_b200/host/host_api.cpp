// extern "C" entry points of libnexd_host.so (declared in include/nexd_host.h).
#include <cstring>
#include <exception>
#include <string>

#include "../../include/nexd_host.h"
#include "mesh_db.hpp"
#include "partition.hpp"

struct nexd_partition {
  std::vector<nexd::PartData> parts;
};

struct nexd_mesh {
  nexd::MeshDB db;
  std::vector<double> src_rst, rec_rst;
  std::vector<int32_t> recnr;
};

namespace {
thread_local std::string g_last_error;

int fail(const std::string& msg) {
  g_last_error = msg;
  return NEXD_ERR_INVALID;
}
}  // namespace

namespace {
nexd::BuildOptions to_options(const nexd_build_opts* opts) {
  nexd::BuildOptions o;
  if (opts) {
    if (opts->N > 0) o.N = opts->N;
    o.timeint = opts->timeint;
    o.cfl = opts->cfl;
    o.nt = opts->nt;
    o.t0 = opts->t0;
    o.stf_stage_time = opts->stf_stage_time;
    o.init_value = opts->init_value;
    o.nbatch = opts->nbatch > 0 ? opts->nbatch : 1;
  }
  return o;
}

template <class Build>
int make_mesh(nexd_mesh** out, Build build) {
  try {
    auto* m = new nexd_mesh;
    try {
      build(m->db);
    } catch (...) {
      delete m;
      throw;
    }
    for (const auto& s : m->db.src) m->src_rst.insert(m->src_rst.end(), s.rst, s.rst + 3);
    for (const auto& r : m->db.rec) {
      m->rec_rst.insert(m->rec_rst.end(), r.rst, r.rst + 3);
      m->recnr.push_back(r.nr);
    }
    *out = m;
    return NEXD_OK;
  } catch (const std::exception& e) {
    return fail(e.what());
  }
}
}  // namespace

extern "C" {

int nexd_mesh_build(const char* dir, const nexd_build_opts* opts, nexd_mesh** out) {
  if (!dir || !out) return fail("nexd_mesh_build: null argument");
  *out = nullptr;
  const nexd::BuildOptions o = to_options(opts);
  return make_mesh(out, [&](nexd::MeshDB& db) { nexd::build_from_directory(dir, o, db); });
}

int nexd_mesh_load_database(const char* dir, const nexd_build_opts* opts, nexd_mesh** out) {
  if (!dir || !out) return fail("nexd_mesh_load_database: null argument");
  *out = nullptr;
  const nexd::BuildOptions o = to_options(opts);
  return make_mesh(out, [&](nexd::MeshDB& db) { nexd::build_from_database(dir, o, db); });
}

int nexd_mesh_write_database(const nexd_mesh* mesh, const char* outdir) {
  if (!mesh || !outdir) return fail("nexd_mesh_write_database: null argument");
  try {
    nexd::write_database(mesh->db, outdir);
    return NEXD_OK;
  } catch (const std::exception& e) {
    return fail(e.what());
  }
}

const nexd_desc* nexd_mesh_desc(const nexd_mesh* mesh) { return mesh ? &mesh->db.desc : nullptr; }

int nexd_mesh_get_info(const nexd_mesh* mesh, nexd_mesh_info* out) {
  if (!mesh || !out) return fail("nexd_mesh_get_info: null argument");
  const auto& db = mesh->db;
  out->dtfactor = db.dtfactor;
  out->dt = db.dt;
  out->minGLL = db.op.minGLL;
  out->cfl = db.par.cfl;
  out->nglob = db.nglob;
  out->ncoord = db.ncoord;
  out->vx = db.vx.data();
  out->vy = db.vy.data();
  out->vz = db.vz.data();
  out->mass = db.mass.data();
  out->vdm = db.V.data();
  out->src_rst = mesh->src_rst.data();
  out->rec_rst = mesh->rec_rst.data();
  out->recnr = mesh->recnr.data();
  out->mu = db.mu.data();
  out->lambda = db.lambda.data();
  out->n_warnings = int32_t(db.warnings.size());
  return NEXD_OK;
}

int nexd_mesh_write_seismograms(const nexd_mesh* mesh, const char* outdir, const float* traces, int32_t nt_written,
                                int32_t batch) {
  if (!mesh || !outdir || !traces) return fail("nexd_mesh_write_seismograms: null argument");
  if (nt_written < 0 || nt_written > mesh->db.par.nt) return fail("nexd_mesh_write_seismograms: bad nt_written");
  if (batch < 0 || batch >= mesh->db.desc.nbatch) return fail("nexd_mesh_write_seismograms: bad batch");
  try {
    nexd::write_seismograms(outdir, mesh->db, traces, nt_written, batch);
    return NEXD_OK;
  } catch (const std::exception& e) {
    return fail(e.what());
  }
}

int nexd_partition_create(const nexd_desc* desc, int32_t nparts, const int32_t* part, const double* centroid,
                          nexd_partition** out) {
  if (!desc || !out) return fail("nexd_partition_create: null argument");
  *out = nullptr;
  if (desc->abi_version != NEXD_ABI_VERSION) return fail("nexd_partition_create: ABI version mismatch");
  try {
    std::vector<int32_t> p;
    if (part) p.assign(part, part + desc->nelem);
    else p = nexd::bisect_partition(centroid, desc->nelem, nparts);
    auto* ps = new nexd_partition;
    try {
      nexd::split_descriptor(*desc, p, nparts, ps->parts);
    } catch (...) {
      delete ps;
      throw;
    }
    *out = ps;
    return NEXD_OK;
  } catch (const std::exception& e) {
    return fail(e.what());
  }
}

int nexd_partition_get(const nexd_partition* ps, int32_t index, nexd_part_view* out) {
  if (!ps || !out) return fail("nexd_partition_get: null argument");
  if (index < 0 || index >= int32_t(ps->parts.size())) return fail("nexd_partition_get: index out of range");
  const nexd::PartData& d = ps->parts[index];
  out->desc = &d.desc;
  out->halo = &d.halo;
  out->nelem = int32_t(d.elem_global.size());
  out->elem_global = d.elem_global.data();
  out->nsrc = int32_t(d.src_global.size());
  out->src_global = d.src_global.data();
  out->nrec = int32_t(d.rec_global.size());
  out->rec_global = d.rec_global.data();
  return NEXD_OK;
}

int nexd_partition_count(const nexd_partition* ps, int32_t* n) {
  if (!ps || !n) return fail("nexd_partition_count: null argument");
  *n = int32_t(ps->parts.size());
  return NEXD_OK;
}

void nexd_partition_free(nexd_partition* ps) { delete ps; }

int nexd_mesh_last_error(char* buf, size_t len) {
  if (!buf || len == 0) return NEXD_ERR_INVALID;
  std::strncpy(buf, g_last_error.c_str(), len - 1);
  buf[len - 1] = '\0';
  return NEXD_OK;
}

void nexd_mesh_free(nexd_mesh* mesh) { delete mesh; }

}  // extern "C"
