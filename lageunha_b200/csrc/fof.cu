// Friends-of-friends groups on the engine's sorted particles and octree.
//
// Reference: pnew_fof_link (FoF/fof.c:217-290) grows a group from a seed,
// linking every particle whose distance to a member is <= fof_link, which
// PreFoF (Cosmos/PreFoF.c:267-385) runs cell by cell with a linking length
// FOF_LINK = 0.2 mean separations and keeps groups of at least FOF_MINNUM =
// 20 members. The groups are the connected components of the "distance <=
// link" relation, so any linking order gives the same partition. Here every
// sorted particle walks the octree of the force evaluation (cubes farther
// than the link are pruned) and joins each linked particle of higher sorted
// index in a lock-free union-find; the roots then count their members, and
// every particle of a group of >= min_members gets the group's smallest
// caller index as its label (-1 otherwise).
#include "ctx.cuh"

using namespace tpm;

namespace {

constexpr int kFofStack = 256;
constexpr int kFofThreads = 128;

TPM_D uint32_t find_root(uint32_t *parent, uint32_t x) {
  uint32_t p = parent[x];
  while (p != x) {
    uint32_t g = parent[p];
    parent[x] = g;  // path halving; racing writers only shorten paths
    x = p;
    p = g;
  }
  return x;
}

TPM_D void unite(uint32_t *parent, uint32_t a, uint32_t b) {
  while (true) {
    a = find_root(parent, a);
    b = find_root(parent, b);
    if (a == b) return;
    if (a > b) {
      uint32_t t = a;
      a = b;
      b = t;
    }
    // hook the larger root under the smaller one, if it is still a root
    uint32_t old = atomicCAS(&parent[b], b, a);
    if (old == b) return;
    b = old;
  }
}

TPM_D float wrapd(uint32_t a, uint32_t b, float cpu) { return (float)(int32_t)(a - b) * cpu; }

__global__ void k_fof_init(uint32_t *parent, uint32_t *gsize, uint32_t *label, int64_t np) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < np; i += (int64_t)gridDim.x * blockDim.x) {
    parent[i] = (uint32_t)i;
    gsize[i] = 0;
    label[i] = 0xffffffffu;
  }
}

// One sorted particle per thread: depth-first over the octree, cubes beyond
// the link pruned, particles of leaves tested against the link.
__global__ void __launch_bounds__(kFofThreads) k_fof_link(const uint32_t *__restrict__ spos, const uint4 *__restrict__ walkA,
                                                          const uint4 *__restrict__ walkB, int64_t np, float cpu,
                                                          float link2, uint32_t *parent, uint32_t *err) {
  uint32_t stack[kFofStack];
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < np; i += (int64_t)gridDim.x * blockDim.x) {
    uint32_t px = spos[3 * i + 0], py = spos[3 * i + 1], pz = spos[3 * i + 2];
    int top = 0;
    stack[top++] = 0u;
    while (top > 0) {
      uint32_t node = stack[--top];
      uint4 geo = walkA[2 * (int64_t)node];
      uint4 rec = walkB[node];
      float half = __uint_as_float(geo.w);
      float dx = fmaxf(fabsf(wrapd(geo.x, px, cpu)) - half, 0.f);
      float dy = fmaxf(fabsf(wrapd(geo.y, py, cpu)) - half, 0.f);
      float dz = fmaxf(fabsf(wrapd(geo.z, pz, cpu)) - half, 0.f);
      if (dx * dx + dy * dy + dz * dz > link2 * 1.0001f + 1e-12f) continue;
      uint32_t nch = rec.w & 0xffffu;
      if (nch == 0) {
        uint32_t s = rec.x, e = rec.x + rec.y;
        for (uint32_t j = (s > (uint32_t)i + 1 ? s : (uint32_t)i + 1); j < e; j++) {
          float ex = wrapd(spos[3 * (int64_t)j + 0], px, cpu);
          float ey = wrapd(spos[3 * (int64_t)j + 1], py, cpu);
          float ez = wrapd(spos[3 * (int64_t)j + 2], pz, cpu);
          if (ex * ex + ey * ey + ez * ez <= link2) unite(parent, (uint32_t)i, j);
        }
      } else {
        if (top + (int)nch > kFofStack) {
          atomicOr(err, (uint32_t)kErrStackOverflow);
          break;
        }
        for (uint32_t k = 0; k < nch; k++) stack[top++] = rec.z + k;
      }
    }
  }
}

// After the links: every particle's root, found without rewriting parent (a
// path-splitting write racing with another thread's could leave an entry on
// an inner node), and the member count of every root.
__global__ void k_fof_count(const uint32_t *__restrict__ parent, uint32_t *root, uint32_t *gsize, int64_t np) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < np; i += (int64_t)gridDim.x * blockDim.x) {
    uint32_t x = (uint32_t)i, p = parent[x];
    while (p != x) {
      x = p;
      p = parent[x];
    }
    root[i] = x;
    atomicAdd(&gsize[x], 1u);
  }
}

__global__ void k_fof_label_min(const uint32_t *root, const uint32_t *gsize, const uint32_t *perm, int64_t np,
                                uint32_t min_members, uint32_t *label, uint32_t *ngroups) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < np; i += (int64_t)gridDim.x * blockDim.x) {
    uint32_t r = root[i];
    if (gsize[r] >= min_members) {
      atomicMin(&label[r], perm[i]);
      if (r == (uint32_t)i) atomicAdd(ngroups, 1u);
    }
  }
}

__global__ void k_fof_scatter(const uint32_t *root, const uint32_t *gsize, const uint32_t *perm, int64_t np,
                              uint32_t min_members, const uint32_t *label, int32_t *out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < np; i += (int64_t)gridDim.x * blockDim.x) {
    uint32_t r = root[i];
    out[perm[i]] = gsize[r] >= min_members ? (int32_t)label[r] : -1;
  }
}

int grid_of(int64_t n) {
  int64_t b = (n + 255) / 256;
  if (b > 148 * 16) b = 148 * 16;
  return (int)(b < 1 ? 1 : b);
}

}  // namespace

extern "C" {

int tpm_fof(tpm_ctx *c, float link, int32_t min_members, int32_t *labels, int mem, int64_t *ngroups) {
  if (!c || !labels || !(link > 0.f) || min_members < 1) return fail(TPM_E_ARG, "bad arguments to tpm_fof");
  if (c->np <= 0) return fail(TPM_E_STATE, "no particles loaded");
  if (2.f * link >= (float)c->prm.n_mesh) return fail(TPM_E_ARG, "link too large for the box");
  CK(cudaSetDevice(c->device));
  cudaStream_t st = c->st;
  int64_t np = c->np;
  // the sort and the octree of a force evaluation (no walk)
  int rc = enqueue_forces(c, TPM_PART_TREE, st, false, false);
  if (rc) return rc;
  // five words per particle, reusing the caller-order force scratch and the
  // alternate sort buffers, which hold nothing between evaluations
  uint32_t *parent = c->val_alt == c->perm ? c->val : c->val_alt;
  uint32_t *gsize = reinterpret_cast<uint32_t *>(c->key_alt == c->skey ? c->key : c->key_alt);
  uint32_t *label = gsize + np;
  int32_t *out = reinterpret_cast<int32_t *>(c->fout);
  uint32_t *root = reinterpret_cast<uint32_t *>(c->fout) + np;
  uint32_t *ng = c->tb.counters + 12;
  CK(cudaMemsetAsync(ng, 0, sizeof(uint32_t), st));
  k_fof_init<<<grid_of(np), 256, 0, st>>>(parent, gsize, label, np);
  int lb = (int)((np + kFofThreads - 1) / kFofThreads);
  if (lb > 148 * 32) lb = 148 * 32;
  float cpu = (float)((double)c->g.n / 4294967296.0);
  k_fof_link<<<lb, kFofThreads, 0, st>>>(c->spos, c->tb.walkA, c->tb.walkB, np, cpu, link * link, parent, c->err);
  k_fof_count<<<grid_of(np), 256, 0, st>>>(parent, root, gsize, np);
  k_fof_label_min<<<grid_of(np), 256, 0, st>>>(root, gsize, c->perm, np, (uint32_t)min_members, label, ng);
  k_fof_scatter<<<grid_of(np), 256, 0, st>>>(root, gsize, c->perm, np, (uint32_t)min_members, label, out);
  CK(cudaGetLastError());
  uint32_t herr = 0, hng = 0;
  CK(cudaMemcpyAsync(&herr, c->err, sizeof(herr), cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(&hng, ng, sizeof(hng), cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(labels, out, sizeof(int32_t) * np,
                     mem == TPM_MEM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  // the scratch buffers were overwritten: no forces are held
  c->parts_valid = 0;
  if (herr) return fail(herr & kErrStackOverflow ? TPM_E_OVERFLOW : TPM_E_CUDA, "device error flags 0x%x", herr);
  if (ngroups) *ngroups = hng;
  return 0;
}

}  // extern "C"
