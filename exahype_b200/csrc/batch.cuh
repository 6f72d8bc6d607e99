// Batched ragged ensemble: many independent uniform-mesh ADER-DG solves
// (different sizes and orders, own time step each) advanced together.
//
// Instances of one (dimension, order, PDE) share a group: their cells are
// concatenated into one set of device arrays (luh, lduh, lQhbnd, lFhbnd) with a
// per-cell instance index, their faces into one face list, so every phase of a
// step is one launch per group whatever the instance sizes. Per-instance time
// scalars (dt, the min-reduction target, t, steps) and cell widths live in
// slot arrays on the device. A step is riemann + boundary + corrector of every
// group, one advance of all instance clocks, then the predictor of every
// group; it is captured once into a CUDA graph and replayed (one graph launch
// per step) until the membership changes.
//
// Membership changes (exa_batch_add / exa_batch_remove) take effect at the
// next exa_batch_commit or exa_batch_step: the affected groups are re-laid out
// (surviving state copied device-to-device), new instances are initialised as
// exa_mesh_init does (admissible step of the initial data, first predictor)
// and the graph is re-captured. Each instance follows exactly the single-mesh
// computation, so its result does not depend on what else is in the batch.
//
// This file is part of capi.cu's translation unit.
#pragma once

namespace exa {

__global__ void batch_advance_kernel(double* dt, double* dtn, double* t, double* steps, const int* live, int nslots) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nslots || !live[i]) return;
  t[i] += dt[i];
  dt[i] = dtn[i];
  dtn[i] = __longlong_as_double(0x7fefffffffffffffll);
  steps[i] += 1.0;
}

// new instances: dt <- admissible step of the initial data, t <- 0, steps <- 0
__global__ void batch_take_dt_kernel(double* dt, double* dtn, double* t, double* steps, const int* slots, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int s = slots[i];
  dt[s] = dtn[s];
  dtn[s] = __longlong_as_double(0x7fefffffffffffffll);
  t[s] = 0.0;
  steps[s] = 0.0;
}

__global__ void batch_reset_kernel(double* dtn, const int* slots, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) dtn[slots[i]] = __longlong_as_double(0x7fefffffffffffffll);
}

}  // namespace exa

struct BatchInst {
  int dim = 0, order = 0, pde = 0, cells[3] = {1, 1, 1}, bc[6] = {0, 0, 0, 0, 0, 0}, ncells = 0;
  double size[3] = {1, 1, 1};
  int group = -1, slot = -1, cell_off = 0;
  bool live = false, removed = false;
  std::vector<double> init;  // initial solution until admitted
};

struct BatchGroup {
  int dim = 0, order = 0, pde = 0, variant = 0;
  exa::KernelSet k{};
  int ncells = 0, nfaces = 0, nb[2] = {0, 0}, boff[2] = {0, 0};
  double *luh = nullptr, *lduh = nullptr, *lQhbnd = nullptr, *lFhbnd = nullptr;
  int *iters = nullptr, *cell_inst = nullptr, *fl = nullptr, *fr = nullptr, *fd = nullptr, *bcell = nullptr,
      *bface = nullptr;
  std::vector<int> members;  // instance ids in layout order
  bool dirty = false;
  bool warmed = false;  // its kernels have run (and set their attributes) outside a capture
};

struct exa_batch {
  std::vector<BatchInst> inst;
  std::vector<BatchGroup> groups;
  int slot_cap = 0;
  double *dt = nullptr, *dtn = nullptr, *t = nullptr, *steps = nullptr, *dx = nullptr;
  int* live = nullptr;
  std::vector<int> slot_owner;  // instance id per slot, -1 free
  unsigned long long* sweeps = nullptr;
  cudaStream_t stream = nullptr;
  bool use_graph = true;
  cudaGraphExec_t graph = nullptr;
  bool graph_valid = false;
};

namespace exa {

static void batch_group_free(BatchGroup& g, cudaStream_t st) {
  for (void* p : {(void*)g.luh, (void*)g.lduh, (void*)g.lQhbnd, (void*)g.lFhbnd, (void*)g.iters, (void*)g.cell_inst,
                  (void*)g.fl, (void*)g.fr, (void*)g.fd, (void*)g.bcell, (void*)g.bface})
    sfree(p, st);
  g.luh = g.lduh = g.lQhbnd = g.lFhbnd = nullptr;
  g.iters = g.cell_inst = g.fl = g.fr = g.fd = g.bcell = g.bface = nullptr;
}

// device bytes one instance adds to its group
static size_t batch_bytes_per_instance(int dim, int order, int npar, long long ncells) {
  const size_t b = order + 1, P = dim == 3 ? b * b * b : b * b, F = dim == 3 ? b * b : b;
  const size_t nV = 5, nD = 5 + npar;
  return (size_t)ncells * (8 * (P * nD + P * nV + 2 * dim * F * (nD + nV)) + 4 * 2 + 4 * 3 * dim) + 64;
}

static int batch_grow_slots(exa_batch* b, int need) {
  if (need <= b->slot_cap) return EXA_OK;
  const int cap = std::max(need, std::max(16, 2 * b->slot_cap));
  double *dt, *dtn, *t, *st, *dx;
  int* live;
  cudaStream_t bs = b->stream;
  if (!salloc(&dt, cap * 8, bs) || !salloc(&dtn, cap * 8, bs) || !salloc(&t, cap * 8, bs) ||
      !salloc(&st, cap * 8, bs) || !salloc(&dx, cap * 24, bs) || !salloc(&live, cap * 4, bs)) {
    cudaGetLastError();
    return fail(EXA_ERR_NOMEM, "exa_batch: slot allocation failed");
  }
  EXA_CUDA(cudaMemsetAsync(live, 0, cap * 4, b->stream));
  EXA_CUDA(cudaMemsetAsync(dx, 0, cap * 24, b->stream));
  if (b->slot_cap) {
    EXA_CUDA(cudaMemcpyAsync(dt, b->dt, b->slot_cap * 8, cudaMemcpyDeviceToDevice, b->stream));
    EXA_CUDA(cudaMemcpyAsync(dtn, b->dtn, b->slot_cap * 8, cudaMemcpyDeviceToDevice, b->stream));
    EXA_CUDA(cudaMemcpyAsync(t, b->t, b->slot_cap * 8, cudaMemcpyDeviceToDevice, b->stream));
    EXA_CUDA(cudaMemcpyAsync(st, b->steps, b->slot_cap * 8, cudaMemcpyDeviceToDevice, b->stream));
    EXA_CUDA(cudaMemcpyAsync(dx, b->dx, b->slot_cap * 24, cudaMemcpyDeviceToDevice, b->stream));
    EXA_CUDA(cudaMemcpyAsync(live, b->live, b->slot_cap * 4, cudaMemcpyDeviceToDevice, b->stream));
  }
  for (void* p : {(void*)b->dt, (void*)b->dtn, (void*)b->t, (void*)b->steps, (void*)b->dx, (void*)b->live})
    sfree(p, bs);
  EXA_CUDA(cudaStreamSynchronize(bs));
  b->dt = dt;
  b->dtn = dtn;
  b->t = t;
  b->steps = st;
  b->dx = dx;
  b->live = live;
  b->slot_owner.resize(cap, -1);
  b->slot_cap = cap;
  b->graph_valid = false;
  return EXA_OK;
}

// New instances of a re-laid-out group (contiguous at its end): upload their
// initial data, then exa_mesh_init's first admissible step and first predictor.
static int batch_init_fresh(exa_batch* b, BatchGroup& ng, const std::vector<int>& fresh,
                            const std::vector<int>& new_off) {
  cudaStream_t st = b->stream;
  const size_t P = ng.k.P, F = ng.k.F, nV = ng.k.nvar, nD = ng.k.nvar + ng.k.npar, D2 = 2 * ng.dim;
  const size_t c0 = (size_t)new_off[fresh.front()], nc = (size_t)ng.ncells - c0;
  std::vector<int> slots;
  for (int id : fresh) {
    const BatchInst& in = b->inst[id];
    EXA_CUDA(cudaMemcpyAsync(ng.luh + (size_t)new_off[id] * P * nD, in.init.data(), in.init.size() * 8,
                             cudaMemcpyHostToDevice, st));
    slots.push_back(in.slot);
  }
  EXA_CUDA(cudaMemsetAsync(ng.lduh + c0 * P * nV, 0, nc * P * nV * 8, st));
  EXA_CUDA(cudaMemsetAsync(ng.lQhbnd + c0 * D2 * F * nD, 0, nc * D2 * F * nD * 8, st));
  EXA_CUDA(cudaMemsetAsync(ng.lFhbnd + c0 * D2 * F * nV, 0, nc * D2 * F * nV * 8, st));
  int* dslots = nullptr;
  if (!salloc(&dslots, slots.size() * 4, st)) {
    cudaGetLastError();
    return fail(EXA_ERR_NOMEM, "exa_batch: device allocation failed");
  }
  const int ns = (int)slots.size();
  int rc = EXA_OK;
  if (cudaMemcpyAsync(dslots, slots.data(), slots.size() * 4, cudaMemcpyHostToDevice, st) != cudaSuccess)
    rc = fail(EXA_ERR_CUDA, "exa_batch: slot upload failed");
  Geometry geo{};
  geo.inst = ng.cell_inst + c0;
  geo.inst_dx = b->dx;
  if (!rc) {
    batch_reset_kernel<<<(ns + 127) / 128, 128, 0, st>>>(b->dtn, dslots, ns);
    rc = ng.k.corrector(ng.luh + c0 * P * nD, nullptr, nullptr, b->dt, b->dtn, geo, (int)nc, nullptr, 0, nullptr, st);
  }
  if (!rc) {
    batch_take_dt_kernel<<<(ns + 127) / 128, 128, 0, st>>>(b->dt, b->dtn, b->t, b->steps, dslots, ns);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) rc = fail(EXA_ERR_CUDA, std::string("exa_batch: ") + cudaGetErrorString(e));
  }
  if (!rc)
    rc = ng.k.predictor(ng.luh + c0 * P * nD, ng.lQhbnd + c0 * D2 * F * nD, ng.lFhbnd + c0 * D2 * F * nV,
                        ng.lduh + c0 * P * nV, ng.iters + c0, b->dt, geo, (int)nc, nullptr, nullptr, PredictorTemps{},
                        false, b->sweeps, ng.variant, st);
  sfree(dslots, st);
  cudaStreamSynchronize(st);
  return rc;
}

// Re-lays out one group: survivors first (state copied), then new instances
// (initial data uploaded, then initialised).
static int batch_relayout(exa_batch* b, BatchGroup& g) {
  cudaStream_t st = b->stream;
  const size_t P = g.k.P, F = g.k.F, nV = g.k.nvar, nD = g.k.nvar + g.k.npar, D2 = 2 * g.dim;
  std::vector<int> keep, fresh;
  for (int id : g.members) {
    const BatchInst& in = b->inst[id];
    if (in.removed) continue;
    (in.live ? keep : fresh).push_back(id);
  }
  // offsets of the live members in the current arrays (member order)
  std::vector<long long> old_off(b->inst.size(), -1);
  {
    long long o = 0;
    for (int id : g.members) {
      old_off[id] = o;
      if (b->inst[id].live) o += b->inst[id].ncells;
    }
  }
  std::vector<int> order = keep;
  order.insert(order.end(), fresh.begin(), fresh.end());
  long long n = 0;
  for (int id : order) n += b->inst[id].ncells;
  if (n > (1ll << 30)) return fail(EXA_ERR_ARG, "exa_batch: too many cells in one group");
  BatchGroup ng = g;
  ng.members = order;
  ng.ncells = (int)n;
  ng.luh = ng.lduh = ng.lQhbnd = ng.lFhbnd = nullptr;
  ng.iters = ng.cell_inst = ng.fl = ng.fr = ng.fd = ng.bcell = ng.bface = nullptr;
  // host-side layout: per-cell instance slots, faces with global cell indices
  std::vector<int> cinst((size_t)n), fl, fr, fd, bcl[2], bfc[2];
  std::vector<int> new_off(b->inst.size(), 0);
  long long off = 0;
  for (int id : order) {
    const BatchInst& in = b->inst[id];
    const int c0 = (int)off;
    new_off[id] = c0;
    for (int c = 0; c < in.ncells; c++) cinst[(size_t)off + c] = in.slot;
    auto cid = [&](int i, int j, int k) { return c0 + (k * in.cells[1] + j) * in.cells[0] + i; };
    for (int k = 0; k < (in.dim == 3 ? in.cells[2] : 1); k++)
      for (int j = 0; j < in.cells[1]; j++)
        for (int i = 0; i < in.cells[0]; i++) {
          const int c = cid(i, j, k);
          int ijk[3] = {i, j, k};
          for (int d = 0; d < in.dim; d++) {
            int nb[3] = {i, j, k};
            nb[d] = ijk[d] + 1;
            if (nb[d] < in.cells[d] || in.bc[2 * d + 1] == EXA_BC_PERIODIC) {
              if (nb[d] >= in.cells[d]) nb[d] = 0;
              fl.push_back(c);
              fr.push_back(cid(nb[0], nb[1], nb[2]));
              fd.push_back(d);
            } else {
              bcl[in.bc[2 * d + 1]].push_back(c);
              bfc[in.bc[2 * d + 1]].push_back(2 * d + 1);
            }
            if (ijk[d] == 0 && in.bc[2 * d] != EXA_BC_PERIODIC) {
              bcl[in.bc[2 * d]].push_back(c);
              bfc[in.bc[2 * d]].push_back(2 * d);
            }
          }
        }
    off += in.ncells;
  }
  ng.nfaces = (int)fl.size();
  std::vector<int> bcell, bface;
  for (int kd = 0; kd < 2; kd++) {
    ng.boff[kd] = (int)bcell.size();
    ng.nb[kd] = (int)bcl[kd].size();
    bcell.insert(bcell.end(), bcl[kd].begin(), bcl[kd].end());
    bface.insert(bface.end(), bfc[kd].begin(), bfc[kd].end());
  }
  const size_t nn = std::max<long long>(n, 1);
  bool ok = salloc(&ng.luh, nn * P * nD * 8, st) && salloc(&ng.lduh, nn * P * nV * 8, st) &&
            salloc(&ng.lQhbnd, nn * D2 * F * nD * 8, st) && salloc(&ng.lFhbnd, nn * D2 * F * nV * 8, st) &&
            salloc(&ng.iters, nn * 4, st) && salloc(&ng.cell_inst, nn * 4, st) &&
            salloc(&ng.fl, std::max<size_t>(1, fl.size()) * 4, st) && salloc(&ng.fr, std::max<size_t>(1, fl.size()) * 4, st) &&
            salloc(&ng.fd, std::max<size_t>(1, fl.size()) * 4, st) &&
            salloc(&ng.bcell, std::max<size_t>(1, bcell.size()) * 4, st) &&
            salloc(&ng.bface, std::max<size_t>(1, bcell.size()) * 4, st);
  if (!ok) {
    cudaGetLastError();
    batch_group_free(ng, st);
    return fail(EXA_ERR_NOMEM, "exa_batch: device allocation failed");
  }
  if (n) EXA_CUDA(cudaMemcpyAsync(ng.cell_inst, cinst.data(), n * 4, cudaMemcpyHostToDevice, st));
  if (!fl.empty()) {
    EXA_CUDA(cudaMemcpyAsync(ng.fl, fl.data(), fl.size() * 4, cudaMemcpyHostToDevice, st));
    EXA_CUDA(cudaMemcpyAsync(ng.fr, fr.data(), fr.size() * 4, cudaMemcpyHostToDevice, st));
    EXA_CUDA(cudaMemcpyAsync(ng.fd, fd.data(), fd.size() * 4, cudaMemcpyHostToDevice, st));
  }
  if (!bcell.empty()) {
    EXA_CUDA(cudaMemcpyAsync(ng.bcell, bcell.data(), bcell.size() * 4, cudaMemcpyHostToDevice, st));
    EXA_CUDA(cudaMemcpyAsync(ng.bface, bface.data(), bface.size() * 4, cudaMemcpyHostToDevice, st));
  }
  // survivors: state copied from the old layout
  for (int id : keep) {
    const size_t src = (size_t)old_off[id], dst = (size_t)new_off[id], nc = b->inst[id].ncells;
    EXA_CUDA(cudaMemcpyAsync(ng.luh + dst * P * nD, g.luh + src * P * nD, nc * P * nD * 8, cudaMemcpyDeviceToDevice, st));
    EXA_CUDA(cudaMemcpyAsync(ng.lduh + dst * P * nV, g.lduh + src * P * nV, nc * P * nV * 8, cudaMemcpyDeviceToDevice, st));
    EXA_CUDA(cudaMemcpyAsync(ng.lQhbnd + dst * D2 * F * nD, g.lQhbnd + src * D2 * F * nD, nc * D2 * F * nD * 8,
                             cudaMemcpyDeviceToDevice, st));
    EXA_CUDA(cudaMemcpyAsync(ng.lFhbnd + dst * D2 * F * nV, g.lFhbnd + src * D2 * F * nV, nc * D2 * F * nV * 8,
                             cudaMemcpyDeviceToDevice, st));
    EXA_CUDA(cudaMemcpyAsync(ng.iters + dst, g.iters + src, nc * 4, cudaMemcpyDeviceToDevice, st));
  }
  int rc = EXA_OK;
  if (!fresh.empty()) {
    rc = batch_init_fresh(b, ng, fresh, new_off);
    ng.warmed = true;  // the first predictor of the new instances ran the group's variant
  }
  if (rc) {
    batch_group_free(ng, st);
    return rc;
  }
  EXA_CUDA(cudaStreamSynchronize(st));
  for (int id : order) b->inst[id].cell_off = new_off[id];
  for (int id : fresh) {
    b->inst[id].live = true;
    std::vector<double>().swap(b->inst[id].init);
  }
  batch_group_free(g, st);
  ng.dirty = false;
  g = ng;
  return EXA_OK;
}

static int batch_apply_changes(exa_batch* b) {
  bool any = false;
  for (BatchGroup& g : b->groups)
    if (g.dirty) {
      int rc = batch_relayout(b, g);
      if (rc) return rc;
      any = true;
    }
  if (!any) return EXA_OK;
  // slots of removed instances are released; live flags follow membership
  std::vector<int> live(b->slot_cap, 0);
  for (BatchInst& in : b->inst) {
    if (in.removed && in.slot >= 0) {
      b->slot_owner[in.slot] = -1;
      in.slot = -1;
      in.live = false;
    } else if (in.live) {
      live[in.slot] = 1;
    }
  }
  EXA_CUDA(cudaMemcpyAsync(b->live, live.data(), b->slot_cap * 4, cudaMemcpyHostToDevice, b->stream));
  EXA_CUDA(cudaStreamSynchronize(b->stream));
  b->graph_valid = false;
  return EXA_OK;
}

// one step of every live instance, launched on b->stream
static int batch_launch_step(exa_batch* b) {
  cudaStream_t st = b->stream;
  int rc;
  for (BatchGroup& g : b->groups) {
    if (g.ncells == 0) continue;
    if ((rc = g.k.riemann(g.lQhbnd, g.lFhbnd, g.fl, g.fr, g.fd, g.nfaces, nullptr, st))) return rc;
    for (int kd = 0; kd < 2; kd++)
      if ((rc = g.k.boundary(g.lQhbnd, g.lFhbnd, g.bcell + g.boff[kd], g.bface + g.boff[kd], g.nb[kd], kd, nullptr,
                             st)))
        return rc;
    Geometry geo{};
    geo.inst = g.cell_inst;
    geo.inst_dx = b->dx;
    if ((rc = g.k.corrector(g.luh, g.lduh, g.lFhbnd, b->dt, b->dtn, geo, g.ncells, nullptr, 1, nullptr, st))) return rc;
  }
  batch_advance_kernel<<<(b->slot_cap + 127) / 128, 128, 0, st>>>(b->dt, b->dtn, b->t, b->steps, b->live, b->slot_cap);
  EXA_LAUNCHED();
  for (BatchGroup& g : b->groups) {
    if (g.ncells == 0) continue;
    Geometry geo{};
    geo.inst = g.cell_inst;
    geo.inst_dx = b->dx;
    if ((rc = g.k.predictor(g.luh, g.lQhbnd, g.lFhbnd, g.lduh, g.iters, b->dt, geo, g.ncells, nullptr, nullptr,
                            PredictorTemps{}, false, b->sweeps, g.variant, st)))
      return rc;
  }
  return EXA_OK;
}

}  // namespace exa

extern "C" {

int exa_batch_create(exa_batch** out) {
  if (!out) return fail(EXA_ERR_ARG, "exa_batch_create: null argument");
  int rc = upload_tables();
  if (rc) return rc;
  std::unique_ptr<exa_batch> b(new exa_batch());
  // the batch holds the many small solves: its blocks are scheduled ahead of
  // those of other streams (large single meshes) when both wait for SMs
  int lo = 0, hi = 0;
  EXA_CUDA(cudaDeviceGetStreamPriorityRange(&lo, &hi));
  EXA_CUDA(cudaStreamCreateWithPriority(&b->stream, cudaStreamNonBlocking, hi));
  if (!salloc(&b->sweeps, 8, b->stream)) {
    cudaGetLastError();
    cudaStreamDestroy(b->stream);
    return fail(EXA_ERR_NOMEM, "exa_batch_create: device allocation failed");
  }
  EXA_CUDA(cudaMemsetAsync(b->sweeps, 0, 8, b->stream));
  rc = batch_grow_slots(b.get(), 16);
  if (rc) return rc;
  *out = b.release();
  return EXA_OK;
}

int exa_batch_destroy(exa_batch* b) {
  if (!b) return EXA_OK;
  if (b->stream) cudaStreamSynchronize(b->stream);
  if (b->graph) cudaGraphExecDestroy(b->graph);
  for (BatchGroup& g : b->groups) batch_group_free(g, b->stream);
  for (void* p : {(void*)b->dt, (void*)b->dtn, (void*)b->t, (void*)b->steps, (void*)b->dx, (void*)b->live,
                  (void*)b->sweeps})
    sfree(p, b->stream);
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
  return EXA_OK;
}

int exa_batch_set_variant(exa_batch* b, int dim, int order, int pde, int variant) {
  if (!b || variant < 0 || variant >= kAllVariants) return fail(EXA_ERR_ARG, "exa_batch_set_variant: bad argument");
  for (BatchGroup& g : b->groups)
    if (g.dim == dim && g.order == order && g.pde == pde) {
      if (g.variant != variant) g.warmed = false;
      g.variant = variant;
      b->graph_valid = false;
      return EXA_OK;
    }
  // no instance of this order yet: its group starts with the given variant
  KernelSet k{};
  if (!find_kernels(dim, order, pde, &k))
    return fail(EXA_ERR_UNSUPPORTED, "exa_batch_set_variant: no kernels built for that dimension/order/PDE");
  BatchGroup g;
  g.dim = dim;
  g.order = order;
  g.pde = pde;
  g.k = k;
  g.variant = variant;
  b->groups.push_back(g);
  return EXA_OK;
}

int exa_batch_get_variant(const exa_batch* b, int dim, int order, int pde, int* variant) {
  if (!b || !variant) return fail(EXA_ERR_ARG, "exa_batch_get_variant: null argument");
  for (const BatchGroup& g : b->groups)
    if (g.dim == dim && g.order == order && g.pde == pde) {
      *variant = g.variant;
      return EXA_OK;
    }
  return fail(EXA_ERR_ARG, "exa_batch_get_variant: no instance of that dimension/order/PDE was added");
}

int exa_batch_add(exa_batch* b, int dim, int order, int pde, const int* cells, const double* size, const int* bc,
                  const double* luh_host, int* id) {
  if (!b || !cells || !size || !bc || !luh_host || !id) return fail(EXA_ERR_ARG, "exa_batch_add: null argument");
  if (dim != 2 && dim != 3) return fail(EXA_ERR_ARG, "exa_batch_add: dim must be 2 or 3");
  KernelSet k{};
  if (!find_kernels(dim, order, pde, &k))
    return fail(EXA_ERR_UNSUPPORTED, "exa_batch_add: no kernels built for dim=" + std::to_string(dim) +
                                         " order=" + std::to_string(order) + " pde=" + std::to_string(pde));
  if (k.linear) return fail(EXA_ERR_UNSUPPORTED, "exa_batch_add: linear PDEs are stepped by exa_mesh only");
  BatchInst in;
  in.dim = dim;
  in.order = order;
  in.pde = pde;
  long long nc = 1;
  for (int d = 0; d < dim; d++) {
    if (cells[d] < 1 || !(size[d] > 0)) return fail(EXA_ERR_ARG, "exa_batch_add: cells >= 1 and size > 0 per axis");
    const bool pl = bc[2 * d] == EXA_BC_PERIODIC, pr = bc[2 * d + 1] == EXA_BC_PERIODIC;
    if (pl != pr) return fail(EXA_ERR_ARG, "exa_batch_add: periodic must be set on both faces of an axis");
    for (int f = 0; f < 2; f++) {
      const int kd = bc[2 * d + f];
      if (kd != EXA_BC_PERIODIC && kd != EXA_BC_OUTFLOW && kd != EXA_BC_REFLECTIVE)
        return fail(EXA_ERR_ARG, "exa_batch_add: unknown boundary kind");
      in.bc[2 * d + f] = kd;
    }
    in.cells[d] = cells[d];
    in.size[d] = size[d];
    nc *= cells[d];
  }
  if (nc > (1ll << 28)) return fail(EXA_ERR_ARG, "exa_batch_add: too many cells");
  in.ncells = (int)nc;
  in.init.assign(luh_host, luh_host + (size_t)nc * k.P * (k.nvar + k.npar));
  int gi = -1;
  for (size_t i = 0; i < b->groups.size(); i++)
    if (b->groups[i].dim == dim && b->groups[i].order == order && b->groups[i].pde == pde) gi = (int)i;
  if (gi < 0) {  // first instance of this order: the autotuner picks its predictor variant
    BatchGroup g;
    g.dim = dim;
    g.order = order;
    g.pde = pde;
    g.k = k;
    exa_solver tmp{k};
    int chosen = 0;
    int rc = exa_solver_autotune(&tmp, 4096, nullptr, &chosen);
    if (rc) return rc;
    g.variant = chosen;
    b->groups.push_back(g);
    gi = (int)b->groups.size() - 1;
  }
  int slot = -1;
  for (int s = 0; s < b->slot_cap; s++)
    if (b->slot_owner[s] < 0) {
      slot = s;
      break;
    }
  if (slot < 0) {
    slot = b->slot_cap;
    int rc = batch_grow_slots(b, b->slot_cap + 1);
    if (rc) return rc;
  }
  in.group = gi;
  in.slot = slot;
  const int new_id = (int)b->inst.size();
  b->slot_owner[slot] = new_id;
  double dx[3] = {1.0, 1.0, 1.0};
  for (int d = 0; d < dim; d++) dx[d] = in.size[d] / in.cells[d];
  EXA_CUDA(cudaMemcpyAsync(b->dx + 3 * slot, dx, 24, cudaMemcpyHostToDevice, b->stream));
  EXA_CUDA(cudaStreamSynchronize(b->stream));
  b->inst.push_back(std::move(in));
  b->groups[gi].members.push_back(new_id);
  b->groups[gi].dirty = true;
  *id = new_id;
  return EXA_OK;
}

int exa_batch_remove(exa_batch* b, int id) {
  if (!b || id < 0 || id >= (int)b->inst.size() || b->inst[id].removed)
    return fail(EXA_ERR_ARG, "exa_batch_remove: unknown instance");
  b->inst[id].removed = true;
  b->groups[b->inst[id].group].dirty = true;
  return EXA_OK;
}

int exa_batch_commit(exa_batch* b) {
  if (!b) return fail(EXA_ERR_ARG, "exa_batch_commit: null batch");
  return batch_apply_changes(b);
}

int exa_batch_set_graph(exa_batch* b, int on) {
  if (!b) return fail(EXA_ERR_ARG, "exa_batch_set_graph: null batch");
  b->use_graph = on != 0;
  b->graph_valid = false;
  return EXA_OK;
}

int exa_batch_step(exa_batch* b, int nsteps) {
  if (!b) return fail(EXA_ERR_ARG, "exa_batch_step: null batch");
  int rc = batch_apply_changes(b);
  if (rc) return rc;
  for (int s = 0; s < nsteps; s++) {
    if (!b->use_graph) {
      if ((rc = batch_launch_step(b))) return rc;
      continue;
    }
    if (b->graph_valid) {
      EXA_CUDA(cudaGraphLaunch(b->graph, b->stream));
      continue;
    }
    if (b->graph) {
      cudaGraphExecDestroy(b->graph);
      b->graph = nullptr;
    }
    bool warm = true;
    for (const BatchGroup& g : b->groups) warm = warm && (g.ncells == 0 || g.warmed);
    if (!warm) {  // run this step eagerly: kernels set their attributes outside any capture
      if ((rc = batch_launch_step(b))) return rc;
      for (BatchGroup& g : b->groups) g.warmed = true;
      continue;
    }
    cudaGraph_t g = nullptr;
    EXA_CUDA(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    rc = batch_launch_step(b);
    const cudaError_t e = cudaStreamEndCapture(b->stream, &g);
    if (rc) {
      if (g) cudaGraphDestroy(g);
      return rc;
    }
    if (e != cudaSuccess) return fail(EXA_ERR_CUDA, std::string("exa_batch_step: capture: ") + cudaGetErrorString(e));
    const cudaError_t e2 = cudaGraphInstantiate(&b->graph, g, 0);
    cudaGraphDestroy(g);
    if (e2 != cudaSuccess)
      return fail(EXA_ERR_CUDA, std::string("exa_batch_step: instantiate: ") + cudaGetErrorString(e2));
    b->graph_valid = true;
    EXA_CUDA(cudaGraphLaunch(b->graph, b->stream));
  }
  return EXA_OK;
}

int exa_batch_state(exa_batch* b, int id, double* t, double* dt, long long* steps) {
  if (!b || id < 0 || id >= (int)b->inst.size()) return fail(EXA_ERR_ARG, "exa_batch_state: unknown instance");
  const BatchInst& in = b->inst[id];
  if (!in.live || in.removed) return fail(EXA_ERR_STATE, "exa_batch_state: instance not live (commit or step first)");
  double h[3];
  EXA_CUDA(cudaMemcpyAsync(&h[0], b->t + in.slot, 8, cudaMemcpyDeviceToHost, b->stream));
  EXA_CUDA(cudaMemcpyAsync(&h[1], b->dt + in.slot, 8, cudaMemcpyDeviceToHost, b->stream));
  EXA_CUDA(cudaMemcpyAsync(&h[2], b->steps + in.slot, 8, cudaMemcpyDeviceToHost, b->stream));
  EXA_CUDA(cudaStreamSynchronize(b->stream));
  if (t) *t = h[0];
  if (dt) *dt = h[1];
  if (steps) *steps = (long long)h[2];
  return EXA_OK;
}

int exa_batch_get_solution(exa_batch* b, int id, double* luh_host) {
  if (!b || !luh_host || id < 0 || id >= (int)b->inst.size())
    return fail(EXA_ERR_ARG, "exa_batch_get_solution: bad argument");
  const BatchInst& in = b->inst[id];
  if (!in.live || in.removed) return fail(EXA_ERR_STATE, "exa_batch_get_solution: instance not live");
  const BatchGroup& g = b->groups[in.group];
  const size_t per = (size_t)g.k.P * (g.k.nvar + g.k.npar);
  EXA_CUDA(cudaMemcpyAsync(luh_host, g.luh + (size_t)in.cell_off * per, (size_t)in.ncells * per * 8,
                           cudaMemcpyDeviceToHost, b->stream));
  EXA_CUDA(cudaStreamSynchronize(b->stream));
  return EXA_OK;
}

int exa_batch_instance_bytes(int dim, int order, int pde, const int* cells, size_t* bytes) {
  if (!cells || !bytes || (dim != 2 && dim != 3)) return fail(EXA_ERR_ARG, "exa_batch_instance_bytes: bad argument");
  long long nc = 1;
  for (int d = 0; d < dim; d++) nc *= std::max(1, cells[d]);
  *bytes = batch_bytes_per_instance(dim, order, pde == EXA_PDE_EULER_TEST ? 1 : 0, nc);
  return EXA_OK;
}

int exa_batch_device_bytes(const exa_batch* b, size_t* bytes) {
  if (!b || !bytes) return fail(EXA_ERR_ARG, "exa_batch_device_bytes: null argument");
  size_t s = (size_t)b->slot_cap * (8 * 4 + 24 + 4) + 8;
  for (const BatchGroup& g : b->groups) {
    long long n = 0;
    for (int id : g.members)
      if (!b->inst[id].removed) n += b->inst[id].ncells;
    s += batch_bytes_per_instance(g.dim, g.order, g.k.npar, n);
  }
  *bytes = s;
  return EXA_OK;
}

int exa_batch_sweeps(exa_batch* b, long long* sweeps) {
  if (!b || !sweeps) return fail(EXA_ERR_ARG, "exa_batch_sweeps: null argument");
  unsigned long long v = 0;
  EXA_CUDA(cudaMemcpyAsync(&v, b->sweeps, 8, cudaMemcpyDeviceToHost, b->stream));
  EXA_CUDA(cudaStreamSynchronize(b->stream));
  *sweeps = (long long)v;
  return EXA_OK;
}

int exa_batch_synchronize(exa_batch* b) {
  if (!b) return fail(EXA_ERR_ARG, "exa_batch_synchronize: null batch");
  EXA_CUDA(cudaStreamSynchronize(b->stream));
  return EXA_OK;
}

int exa_batch_stream(exa_batch* b, void** stream) {
  if (!b || !stream) return fail(EXA_ERR_ARG, "exa_batch_stream: null argument");
  *stream = (void*)b->stream;
  return EXA_OK;
}

}  // extern "C"
