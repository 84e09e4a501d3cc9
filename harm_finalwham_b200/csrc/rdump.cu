// rdump.cu -- the reference's restart dump ("rdump") written from and read
// into device state.
//
// Format (restart_write restart.c:206-235 -> dump_gen dumpgen.c:245-283 ->
// rdump_content restart.c:240-245 -> myfwrite mpi_fileio.c:2073-2150, one
// process, mpicombine 0, no column split):
//   * the header, write_restart_header (restart.c:640-800): host state the
//     device does not own (t, tf, nstep, the options, the coordinate
//     parameters, the cumulative diagnostics ...).  The caller passes its
//     bytes; in text mode it is one line ending in '\n'.
//   * every active zone in DUMPGENLOOP order (global.h:1411-1432: k outer,
//     then j, i fastest), each p[0..7] then unew[0..7]: in text mode
//     (TEXTOUTPUT, the reference's setting without MPI, initbase.c:237) each
//     value as "%21.15g " and '\n' after each zone; in binary mode the 16
//     doubles in host byte order.
// The text of the body is formatted in parallel (blocks of zones, one
// thread per block) and written in order, so the file is exactly what one
// sequential fprintf loop writes.
#include <errno.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <string>
#include <thread>
#include <vector>

#include "harmgpu.h"

const hgpu_config *hg_config(const hgpu_ctx *x, int *is_batch);
extern "C" void hg_set_error(const char *msg);

namespace {

constexpr int kNPR = 8;
constexpr long long kBlock = 16384;  // zones per formatting block

struct Layout {
  int n[4], g[4], nt[4];
  long long nz() const { return (long long)nt[1] * nt[2] * nt[3]; }
  long long zone(int i, int j, int k) const {
    return ((long long)(i + g[1]) * nt[2] + (j + g[2])) * nt[3] + (k + g[3]);
  }
  long long active() const { return (long long)n[1] * n[2] * n[3]; }
  // active zone number a in DUMPGENLOOP order -> (i, j, k)
  void ijk(long long a, int *i, int *j, int *k) const {
    *i = (int)(a % n[1]);
    a /= n[1];
    *j = (int)(a % n[2]);
    *k = (int)(a / n[2]);
  }
};

int layout_of(hgpu_ctx *ctx, Layout *L) {
  int batch = 0;
  const hgpu_config *c = hg_config(ctx, &batch);
  if (batch) {
    hg_set_error("restart dumps are defined for one grid, not for a batch of 1D instances");
    return HGPU_E_INVALID;
  }
  L->n[1] = c->n1;
  L->n[2] = c->n2;
  L->n[3] = c->n3;
  for (int d = 1; d <= 3; d++) {
    L->g[d] = L->n[d] > 1 ? c->ng : 0;
    L->nt[d] = L->n[d] + 2 * L->g[d];
  }
  return HGPU_OK;
}

void format_block(const Layout &L, const double *p, const double *u, long long a0, long long a1, std::string *out) {
  char buf[64];
  out->clear();
  out->reserve((size_t)(a1 - a0) * (2 * kNPR * 22 + 1));
  for (long long a = a0; a < a1; a++) {
    int i, j, k;
    L.ijk(a, &i, &j, &k);
    const long long z = L.zone(i, j, k);
    for (int half = 0; half < 2; half++) {
      const double *v = (half ? u : p) + kNPR * z;
      for (int pl = 0; pl < kNPR; pl++) {
        int len = snprintf(buf, sizeof(buf), "%21.15g ", v[pl]);
        out->append(buf, (size_t)len);
      }
    }
    out->push_back('\n');
  }
}

struct HostState {
  double *p = nullptr, *u = nullptr;
  ~HostState() {
    if (p) hgpu_free_pinned(p);
    if (u) hgpu_free_pinned(u);
  }
  int alloc(long long nz) {
    if (hgpu_alloc_pinned(sizeof(double) * kNPR * nz, (void **)&p) != HGPU_OK ||
        hgpu_alloc_pinned(sizeof(double) * kNPR * nz, (void **)&u) != HGPU_OK)
      return HGPU_E_CUDA;
    return HGPU_OK;
  }
};

int io_error(const char *what, const char *path) {
  char msg[512];
  snprintf(msg, sizeof(msg), "%s %s: %s", what, path, strerror(errno));
  hg_set_error(msg);
  return HGPU_E_INVALID;
}

}  // namespace

extern "C" int hgpu_write_rdump(hgpu_ctx *ctx, const char *path, const void *header, size_t header_bytes,
                                int binary) {
  if (!ctx || !path || (header_bytes && !header)) return HGPU_E_INVALID;
  Layout L;
  int rc = layout_of(ctx, &L);
  if (rc) return rc;
  HostState h;
  if ((rc = h.alloc(L.nz()))) return rc;
  double t, dt;
  if ((rc = hgpu_download_state(ctx, h.p, nullptr, &t, &dt))) return rc;
  if ((rc = hgpu_download_conserved(ctx, h.u))) return rc;

  FILE *f = fopen(path, "wb");
  if (!f) return io_error("cannot open", path);
  bool ok = header_bytes == 0 || fwrite(header, 1, header_bytes, f) == header_bytes;
  const long long na = L.active();
  if (ok && binary) {
    double rec[2 * kNPR];
    for (long long a = 0; a < na && ok; a++) {
      int i, j, k;
      L.ijk(a, &i, &j, &k);
      const long long z = L.zone(i, j, k);
      memcpy(rec, h.p + kNPR * z, sizeof(double) * kNPR);
      memcpy(rec + kNPR, h.u + kNPR * z, sizeof(double) * kNPR);
      ok = fwrite(rec, sizeof(double), 2 * kNPR, f) == 2 * kNPR;
    }
  } else if (ok) {
    const int nthreads = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
    std::vector<std::string> blocks(nthreads);
    for (long long a0 = 0; a0 < na && ok; a0 += kBlock * nthreads) {
      std::vector<std::thread> pool;
      int used = 0;
      for (int b = 0; b < nthreads; b++) {
        const long long s = a0 + kBlock * b;
        if (s >= na) break;
        const long long e = std::min(na, s + kBlock);
        pool.emplace_back(format_block, std::cref(L), h.p, h.u, s, e, &blocks[b]);
        used++;
      }
      for (auto &th : pool) th.join();
      for (int b = 0; b < used && ok; b++) ok = fwrite(blocks[b].data(), 1, blocks[b].size(), f) == blocks[b].size();
    }
  }
  if (fclose(f) != 0) ok = false;
  if (!ok) return io_error("cannot write", path);
  return HGPU_OK;
}

extern "C" int hgpu_read_rdump(hgpu_ctx *ctx, const char *path, size_t header_bytes, int binary, double t,
                               double dt) {
  if (!ctx || !path) return HGPU_E_INVALID;
  Layout L;
  int rc = layout_of(ctx, &L);
  if (rc) return rc;
  HostState h;
  if ((rc = h.alloc(L.nz()))) return rc;
  double t0, dt0;
  // the ghost zones of both arrays are replaced below (bound_prim; unew is
  // defined on active zones only), the active zones by the file
  if ((rc = hgpu_download_state(ctx, h.p, nullptr, &t0, &dt0))) return rc;
  memset(h.u, 0, sizeof(double) * kNPR * L.nz());

  FILE *f = fopen(path, "rb");
  if (!f) return io_error("cannot open", path);
  bool ok = true;
  if (header_bytes) ok = fseek(f, (long)header_bytes, SEEK_SET) == 0;
  const long long na = L.active();
  for (long long a = 0; a < na && ok; a++) {
    int i, j, k;
    L.ijk(a, &i, &j, &k);
    const long long z = L.zone(i, j, k);
    double rec[2 * kNPR];
    if (binary) {
      ok = fread(rec, sizeof(double), 2 * kNPR, f) == 2 * kNPR;
    } else {
      for (int q = 0; q < 2 * kNPR && ok; q++) ok = fscanf(f, "%lf", &rec[q]) == 1;
    }
    if (ok) {
      memcpy(h.p + kNPR * z, rec, sizeof(double) * kNPR);
      memcpy(h.u + kNPR * z, rec + kNPR, sizeof(double) * kNPR);
    }
  }
  fclose(f);
  if (!ok) {
    char msg[512];
    snprintf(msg, sizeof(msg), "%s: short or malformed restart dump (expected %lld zones x 16 values)", path, na);
    hg_set_error(msg);
    return HGPU_E_INVALID;
  }
  // restart_init (restart.c:1-180): the state read, then bound_prim; the
  // conserved state as read (the finite-volume scheme evolves it)
  std::vector<int> noflags((size_t)L.nz(), 0);
  if ((rc = hgpu_upload_state(ctx, h.p, noflags.data(), t, dt))) return rc;
  if ((rc = hgpu_bound_prim(ctx, 0))) return rc;
  if ((rc = hgpu_upload_conserved(ctx, h.u))) return rc;
  return HGPU_OK;
}
