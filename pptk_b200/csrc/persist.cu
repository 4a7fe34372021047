// Tree persistence: a built tree (single tree or forest) written to one
// self-describing host buffer and read back onto a device without a rebuild.
// The reference keeps trees only in process memory (a PyCapsule,
// kdtree_wrapper.cpp:57-74); this has no counterpart there.
//
// Layout: Header, then the sections in order, each padded to 64 bytes:
// tree-ordered points, forward map, records, traversal nodes, per-cloud root
// record, root node, valid offsets, input offsets.  The header carries the
// element counts and an FNV-1a hash of everything after it.  Loading checks
// the header, the sizes and the hash on the host, the records on the host,
// and every node reference, point id and map entry on the device before the
// tree is handed out, so a damaged buffer is an error, never an out-of-range
// read by a query.
#include <cstring>
#include <vector>

#include "build.cuh"
#include "common.cuh"
#include "persist.cuh"
#include "util.cuh"

namespace pptkg {

namespace {

constexpr char MAGIC[8] = {'P', 'P', 'T', 'K', 'G', 'T', 'R', '1'};
constexpr int VERSION = 1;

struct Header {
  char magic[8];
  int32_t version, dtype, rec_dtype, dim;
  int64_t n, nv;
  int32_t n_recs, n_tnodes, depth, tdepth, bucket, max_leaf, ncloud, pad0;
  double empty_split;
  double root_lo[4], root_hi[4];
  int64_t sec_bytes[8];
  uint64_t hash;  // FNV-1a of every byte after the header
};

// FNV-1a over 8-byte words (then the tail bytes): a damage check, not a
// cryptographic one.
uint64_t fnv1a(const char* p, size_t n) {
  uint64_t h = 1469598103934665603ull;
  size_t i = 0;
  for (; i + 8 <= n; i += 8) {
    uint64_t w;
    memcpy(&w, p + i, 8);
    h ^= w;
    h *= 1099511628211ull;
  }
  for (; i < n; i++) {
    h ^= (unsigned char)p[i];
    h *= 1099511628211ull;
  }
  return h;
}

size_t pad64(size_t b) { return (b + 63) / 64 * 64; }

template <typename F>
void with_types(int dtype, int rec_dtype, int dim, F&& f) {
  auto on_rec = [&](auto tq) {
    auto on_dim = [&](auto tr) {
      if (dim == 2)
        f(tq, tr, std::integral_constant<int, 2>());
      else if (dim == 3)
        f(tq, tr, std::integral_constant<int, 3>());
      else if (dim == 4)
        f(tq, tr, std::integral_constant<int, 4>());
      else
        throw Error(E_INVALID, "stored tree: dim must be 2, 3 or 4");
    };
    switch (rec_dtype) {
      case F32: on_dim(float()); break;
      case F64: on_dim(double()); break;
      case I8: on_dim(int8_t()); break;
      case I16: on_dim(int16_t()); break;
      case I32: on_dim(int32_t()); break;
      case I64: on_dim(int64_t()); break;
      case U8: on_dim(uint8_t()); break;
      case U16: on_dim(uint16_t()); break;
      case U32: on_dim(uint32_t()); break;
      case U64: on_dim(uint64_t()); break;
      default: throw Error(E_INVALID, "stored tree: unknown point type");
    }
  };
  if (dtype == F32)
    on_rec(float());
  else if (dtype == F64)
    on_rec(double());
  else
    throw Error(E_INVALID, "stored tree: traversal data must be float32 or float64");
}

// Expected byte sizes of the eight sections.
void section_bytes(int dtype, int rec_dtype, int dim, int64_t n, int64_t nv, int n_recs, int n_tnodes, int ncloud,
                   int64_t out[8]) {
  with_types(dtype, rec_dtype, dim, [&](auto tq, auto tr, auto d) {
    typedef decltype(tq) Tq;
    typedef decltype(tr) Tr;
    constexpr int D = decltype(d)::value;
    out[0] = nv * (int64_t)sizeof(PointRec<Tq, D>);
    out[1] = n * 4;
    out[2] = (int64_t)n_recs * (int64_t)sizeof(Rec<Tr, D>);
    out[3] = (int64_t)n_tnodes * (int64_t)sizeof(TNode<Tq, D>);
    out[4] = (int64_t)ncloud * 4;
    out[5] = (int64_t)ncloud * 4;
    out[6] = (int64_t)(ncloud + 1) * 8;
    out[7] = (int64_t)(ncloud + 1) * 8;
  });
}

// Device check of a loaded tree's references; any failure sets *bad.
template <typename Tq, int D>
__global__ void k_check_tree(const PointRec<Tq, D>* pts, int64_t nv, int64_t n, const int* fwd,
                             const TNode<Tq, D>* nodes, int n_nodes, int* bad) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < nv) {
    const int id = pts[i].id;
    if (id < 0 || id >= n) atomicExch(bad, 1);
  }
  if (i < n) {
    const int p = fwd[i];
    if (p < -1 || p >= nv) atomicExch(bad, 1);
  }
  if (i < n_nodes) {
    for (int c = 0; c < 2; c++) {
      const int ref = nodes[i].ref[c], cnt = nodes[i].cnt[c];
      if (cnt < 0) atomicExch(bad, 1);
      if (cnt == 0) continue;
      if (ref >= 0) {
        if (ref >= n_nodes) atomicExch(bad, 1);
      } else {
        const long long b = -(long long)ref - 1;
        if (b + cnt > nv) atomicExch(bad, 1);
      }
    }
  }
}

}  // namespace

std::vector<char> save_tree(const TreeBase* t, cudaStream_t st) {
  Header h;
  memset(&h, 0, sizeof(h));
  memcpy(h.magic, MAGIC, 8);
  h.version = VERSION;
  h.dtype = t->dtype;
  h.rec_dtype = t->rec_dtype;
  h.dim = t->dim;
  h.n = t->n;
  h.nv = t->nv;
  h.n_recs = t->n_recs;
  h.n_tnodes = t->n_tnodes;
  h.depth = t->depth;
  h.tdepth = t->tdepth;
  h.bucket = t->bucket;
  h.max_leaf = t->max_leaf;
  h.ncloud = t->ncloud;
  h.empty_split = t->empty_split;
  for (int d = 0; d < 4; d++) {
    h.root_lo[d] = t->root_lo[d];
    h.root_hi[d] = t->root_hi[d];
  }
  section_bytes(h.dtype, h.rec_dtype, h.dim, h.n, h.nv, h.n_recs, h.n_tnodes, h.ncloud, h.sec_bytes);
  const void* src[8] = {t->pts, t->fwd, t->recs, t->tnodes, t->root_rec, t->root_tnode, t->valid_off, t->orig_off};
  size_t total = sizeof(Header);
  for (int s = 0; s < 8; s++) total += pad64((size_t)h.sec_bytes[s]);
  std::vector<char> out(total, 0);
  size_t at = sizeof(Header);
  for (int s = 0; s < 8; s++) {
    if (h.sec_bytes[s] > 0) {
      if (!src[s]) throw Error(E_INVALID, "tree has no device data to save");
      PPTKG_CUDA(cudaMemcpyAsync(out.data() + at, src[s], (size_t)h.sec_bytes[s], cudaMemcpyDeviceToHost, st));
    }
    at += pad64((size_t)h.sec_bytes[s]);
  }
  PPTKG_CUDA(cudaStreamSynchronize(st));
  h.hash = fnv1a(out.data() + sizeof(Header), total - sizeof(Header));
  memcpy(out.data(), &h, sizeof(Header));
  return out;
}

TreeBase* load_tree(const char* buf, size_t size, cudaStream_t st) {
  if (!buf || size < sizeof(Header)) throw Error(E_INVALID, "stored tree: buffer too small");
  Header h;
  memcpy(&h, buf, sizeof(Header));
  if (memcmp(h.magic, MAGIC, 8) != 0) throw Error(E_INVALID, "stored tree: not a pptk_b200 tree");
  if (h.version != VERSION) throw Error(E_INVALID, "stored tree: unsupported version " + std::to_string(h.version));
  if (h.n < 0 || h.nv < 0 || h.nv > h.n || h.n > (int64_t)INT32_MAX / 2 || h.n_recs < 0 || h.n_tnodes < 0 ||
      h.ncloud < 1 || h.depth < 0 || h.tdepth < 0 || h.bucket < 1 || h.n_tnodes < h.ncloud)
    throw Error(E_INVALID, "stored tree: inconsistent header");
  int64_t want[8];
  section_bytes(h.dtype, h.rec_dtype, h.dim, h.n, h.nv, h.n_recs, h.n_tnodes, h.ncloud, want);
  size_t total = sizeof(Header);
  for (int s = 0; s < 8; s++) {
    if (h.sec_bytes[s] != want[s]) throw Error(E_INVALID, "stored tree: section sizes do not match the header");
    total += pad64((size_t)want[s]);
  }
  if (size < total) throw Error(E_INVALID, "stored tree: buffer shorter than its sections");
  if (fnv1a(buf + sizeof(Header), total - sizeof(Header)) != h.hash)
    throw Error(E_INVALID, "stored tree: checksum mismatch (damaged data)");
  size_t off[8];
  size_t at = sizeof(Header);
  for (int s = 0; s < 8; s++) {
    off[s] = at;
    at += pad64((size_t)want[s]);
  }
  // host checks of the per-cloud tables and the records
  std::vector<int64_t> valid_off(h.ncloud + 1), orig_off(h.ncloud + 1);
  std::vector<int32_t> root_rec(h.ncloud), root_tnode(h.ncloud);
  memcpy(valid_off.data(), buf + off[6], (size_t)want[6]);
  memcpy(orig_off.data(), buf + off[7], (size_t)want[7]);
  memcpy(root_rec.data(), buf + off[4], (size_t)want[4]);
  memcpy(root_tnode.data(), buf + off[5], (size_t)want[5]);
  if (valid_off[0] != 0 || valid_off[h.ncloud] != h.nv || orig_off[0] != 0 || orig_off[h.ncloud] != h.n)
    throw Error(E_INVALID, "stored tree: bad cloud offsets");
  for (int c = 0; c < h.ncloud; c++) {
    if (valid_off[c + 1] < valid_off[c] || orig_off[c + 1] < orig_off[c])
      throw Error(E_INVALID, "stored tree: bad cloud offsets");
    if (root_rec[c] < -1 || root_rec[c] >= h.n_recs || root_tnode[c] < 0 || root_tnode[c] >= h.n_tnodes)
      throw Error(E_INVALID, "stored tree: bad cloud roots");
  }
  with_types(h.dtype, h.rec_dtype, h.dim, [&](auto tq, auto tr, auto d) {
    typedef decltype(tr) Tr;
    constexpr int D = decltype(d)::value;
    const Rec<Tr, D>* r = reinterpret_cast<const Rec<Tr, D>*>(buf + off[2]);
    std::vector<int32_t> kids(2 * (size_t)h.n_recs);
    for (int i = 0; i < h.n_recs; i++) {
      Rec<Tr, D> x;
      memcpy(&x, r + i, sizeof(x));
      if (x.left < -1 || x.left >= h.n_recs || x.right < -1 || x.right >= h.n_recs || x.begin < 0 ||
          x.end < x.begin || x.end > h.nv || x.split_dim < -1 || x.split_dim >= D || x.ntrim < 0)
        throw Error(E_INVALID, "stored tree: bad record");
      kids[2 * (size_t)i] = x.left;
      kids[2 * (size_t)i + 1] = x.right;
    }
    // the records reachable from the roots must form trees: a record reached
    // twice (a cycle or a shared child) is rejected before anything walks them
    std::vector<char> seen(h.n_recs, 0);
    std::vector<int32_t> stack;
    for (int c = 0; c < h.ncloud; c++) {
      if (root_rec[c] < 0) continue;
      stack.push_back(root_rec[c]);
      while (!stack.empty()) {
        const int32_t v = stack.back();
        stack.pop_back();
        if (seen[v]) throw Error(E_INVALID, "stored tree: records do not form a tree");
        seen[v] = 1;
        for (int j = 0; j < 2; j++)
          if (kids[2 * (size_t)v + j] >= 0) stack.push_back(kids[2 * (size_t)v + j]);
      }
    }
  });
  std::unique_ptr<TreeBase> t(new TreeBase());
  t->stream = st;
  PPTKG_CUDA(cudaGetDevice(&t->device));
  t->dtype = h.dtype;
  t->rec_dtype = h.rec_dtype;
  t->dim = h.dim;
  t->n = h.n;
  t->nv = h.nv;
  t->n_recs = h.n_recs;
  t->n_tnodes = h.n_tnodes;
  t->depth = h.depth;
  t->tdepth = h.tdepth;
  t->bucket = h.bucket;
  t->max_leaf = h.max_leaf;
  t->empty_split = h.empty_split;
  t->ncloud = h.ncloud;
  for (int d = 0; d < 4; d++) {
    t->root_lo[d] = h.root_lo[d];
    t->root_hi[d] = h.root_hi[d];
  }
  t->valid_off_h = valid_off;
  t->orig_off_h = orig_off;
  t->root_tnode_h = root_tnode;
  void** dst[8] = {&t->pts, (void**)&t->fwd, &t->recs, &t->tnodes, (void**)&t->root_rec, (void**)&t->root_tnode,
                   (void**)&t->valid_off, (void**)&t->orig_off};
  for (int s = 0; s < 8; s++) {
    PPTKG_CUDA(dev_malloc(dst[s], std::max<size_t>((size_t)want[s], 1), st));
    if (want[s]) PPTKG_CUDA(cudaMemcpyAsync(*dst[s], buf + off[s], (size_t)want[s], cudaMemcpyHostToDevice, st));
  }
  // device checks of every reference a query follows
  BuildBuf<int> bad(1, st);
  PPTKG_CUDA(cudaMemsetAsync(bad.get(), 0, sizeof(int), st));
  with_types(h.dtype, h.rec_dtype, h.dim, [&](auto tq, auto tr, auto d) {
    typedef decltype(tq) Tq;
    constexpr int D = decltype(d)::value;
    const int64_t work = std::max<int64_t>(std::max<int64_t>(h.nv, h.n), h.n_tnodes);
    if (work > 0) {
      k_check_tree<Tq, D><<<(unsigned)((work + 255) / 256), 256, 0, st>>>(
          (const PointRec<Tq, D>*)t->pts, h.nv, h.n, t->fwd, (const TNode<Tq, D>*)t->tnodes, h.n_tnodes, bad.get());
      PPTKG_CHECK_LAUNCH();
    }
  });
  int hb = 0;
  PPTKG_CUDA(cudaMemcpyAsync(&hb, bad.get(), sizeof(int), cudaMemcpyDeviceToHost, st));
  PPTKG_CUDA(cudaStreamSynchronize(st));
  if (hb) throw Error(E_INVALID, "stored tree: a node, point id or index map entry is out of range");
  return t.release();
}

}  // namespace pptkg
