// mesh.cu -- P1 meshes on the device, equation numbering, the node graph of
// SpMatrix(mesh) and the element-to-CSR scatter map.
//
//   * ofg_mesh_create_rect reproduces Mesh(xmin,..,TRIANGLE)
//     (src/mesh/Mesh.cpp:547-676): the 1-D coordinate ladders are
//     accumulated on the host exactly as the reference accumulates them
//     (x.y += hy per node), so node coordinates are bit-identical.
//   * equations: dof = running count of code-0 nodes (Mesh::NumberEquations
//     with removeImposedDOF, Mesh.cpp:1497-1509), an exclusive scan.
//   * NodeGraph (src/linear_algebra/GraphOfMatrix.cpp:347-375) stores every
//     (dof_i, dof_j) pair of every element, sorts and uniques.  Here each row
//     gathers the DOFs of the elements around its node, sorts and uniques
//     them in registers: same set, same order, no global sort.
//   * node-to-element lists (elements ascending per node), from which the
//     assembly gathers each row in OFELI's element order.
#include <algorithm>
#include <numeric>

#include "internal.cuh"

namespace ofg {
namespace {

constexpr int kMaxGather = 256;  // distinct DOFs per row (matrix row length limit)

__global__ void rect_nodes(int64_t nx, int64_t ny, const double* xs, const double* ys, int cx0,
                           int cxN, int cy0, int cyN, double* xy, int32_t* code)
{
   int64_t nn = (nx + 1) * (ny + 1);
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < nn; k += stride) {
      int64_t i = k / (ny + 1), j = k % (ny + 1);
      int c = 0;
      if (j == 0 && cy0 > 0) c = cy0;
      if (j == ny && cyN > 0) c = cyN;
      if (i == 0 && cx0 > 0) c = cx0;
      if (i == nx && cxN > 0) c = cxN;
      xy[2 * k] = xs[i];
      xy[2 * k + 1] = ys[j];
      code[k] = c;
   }
}

// Cell (i,j), i in 1..nx, j in 1..ny, is visited when node n = i*(ny+1)+j+1
// is created; its triangles are theNodes[n-ny-3], theNodes[n-2],
// theNodes[n-1] and theNodes[n-1], theNodes[n-ny-2], theNodes[n-ny-3].
__global__ void rect_elems(int64_t nx, int64_t ny, int32_t* elem)
{
   int64_t ncell = nx * ny;
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < ncell; c += stride) {
      int64_t i = c / ny + 1, j = c % ny + 1;
      int32_t n = (int32_t)(i * (ny + 1) + j + 1);
      int32_t* e = elem + 6 * c;
      e[0] = n - (int32_t)ny - 3;
      e[1] = n - 2;
      e[2] = n - 1;
      e[3] = n - 1;
      e[4] = n - (int32_t)ny - 2;
      e[5] = n - (int32_t)ny - 3;
   }
}

__global__ void kuhn_nodes(int64_t M, double* xyz, int32_t* code)
{
   int64_t P = M + 1, nn = P * P * P;
   double h = 1.0 / (double)M;
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < nn; k += stride) {
      int64_t ix = k % P, jy = (k / P) % P, kz = k / (P * P);
      xyz[3 * k] = (double)ix * h;
      xyz[3 * k + 1] = (double)jy * h;
      xyz[3 * k + 2] = (double)kz * h;
      code[k] = (ix == 0 || jy == 0 || kz == 0 || ix == M || jy == M || kz == M) ? 1 : 0;
   }
}

// 6 tetrahedra per cell: vertex 0 = cell origin, then one unit step along
// each axis in the order of a permutation; odd permutations swap vertices 1
// and 2 so that every Jacobian is positive.
__global__ void kuhn_elems(int64_t M, int32_t* elem)
{
   const int perm[6][3] = {{0, 1, 2}, {0, 2, 1}, {1, 0, 2}, {1, 2, 0}, {2, 0, 1}, {2, 1, 0}};
   const int odd[6] = {0, 1, 1, 0, 0, 1};
   int64_t P = M + 1, ncell = M * M * M;
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < ncell * 6; t += stride) {
      int64_t cell = t / 6;
      int q = (int)(t % 6);
      int64_t c[3] = {cell % M, (cell / M) % M, cell / (M * M)};
      int32_t v[4];
      v[0] = (int32_t)(c[0] + P * (c[1] + P * c[2]));
      for (int s = 0; s < 3; ++s) {
         c[perm[q][s]]++;
         v[s + 1] = (int32_t)(c[0] + P * (c[1] + P * c[2]));
      }
      if (odd[q]) { int32_t tmp = v[1]; v[1] = v[2]; v[2] = tmp; }
      for (int s = 0; s < 4; ++s) elem[4 * t + s] = v[s];
   }
}

__global__ void free_flags(int64_t nn, const int32_t* code, int64_t* flag)
{
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nn; i += stride)
      flag[i] = code[i] == 0 ? 1 : 0;
}

__global__ void number_dofs(int64_t nn, const int32_t* code, const int64_t* prefix, int32_t* dof)
{
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nn; i += stride)
      dof[i] = code[i] == 0 ? (int32_t)(prefix[i] + 1) : 0;
}

__global__ void check_elems(int64_t ne, int nen, int64_t nn, const int32_t* elem, int* bad)
{
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < ne * nen; k += stride)
      if (elem[k] < 0 || elem[k] >= nn) atomicOr(bad, 1);
}

__global__ void count_n2e(int64_t ne, int nen, const int32_t* elem, int64_t* cnt)
{
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < ne * nen; k += stride)
      atomicAdd((unsigned long long*)&cnt[elem[k]], 1ULL);
}

__global__ void fill_n2e(int64_t ne, int nen, const int32_t* elem, const int64_t* start,
                         int32_t* cursor, int32_t* n2e)
{
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < ne * nen; k += stride) {
      int32_t node = elem[k];
      int32_t slot = atomicAdd(&cursor[node], 1);
      n2e[start[node] + slot] = (int32_t)(k / nen);
   }
}

__global__ void finish_n2e(int64_t nn, const int64_t* start, int32_t* ptr32, int32_t* n2e)
{
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i <= nn; i += stride) {
      ptr32[i] = (int32_t)start[i];
      if (i == nn) continue;
      // insertion sort of the (short) element list of node i
      int64_t b = start[i], e = start[i + 1];
      for (int64_t p = b + 1; p < e; ++p) {
         int32_t v = n2e[p];
         int64_t q = p - 1;
         while (q >= b && n2e[q] > v) { n2e[q + 1] = n2e[q]; --q; }
         n2e[q + 1] = v;
      }
   }
}

// Row gather of NodeGraph: sorted unique DOFs of all elements around node i.
// pass 0 counts, pass 1 writes 0-based columns.
__global__ void node_graph_rows(int64_t nn, int nen, const int32_t* elem, const int32_t* dof,
                                const int32_t* n2e_ptr, const int32_t* n2e, int64_t* rowlen,
                                const int32_t* row_ptr, int32_t* col, int pass, int* overflow)
{
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   int32_t buf[kMaxGather];
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nn; i += stride) {
      int32_t r = dof[i];
      if (!r) continue;
      int m = 0;
      for (int32_t p = n2e_ptr[i]; p < n2e_ptr[i + 1]; ++p) {
         const int32_t* en = elem + (int64_t)n2e[p] * nen;
         for (int a = 0; a < nen; ++a) {
            int32_t c = dof[en[a]];
            if (!c) continue;
            // insertion into the sorted buffer, dropping duplicates
            int q = m - 1;
            bool dup = false;
            while (q >= 0 && buf[q] >= c) {
               if (buf[q] == c) { dup = true; break; }
               --q;
            }
            if (dup) continue;
            if (m >= kMaxGather) { atomicOr(overflow, 1); continue; }
            for (int s = m; s > q + 1; --s) buf[s] = buf[s - 1];
            buf[q + 1] = c;
            ++m;
         }
      }
      if (pass == 0) rowlen[r - 1] = m;
      else {
         int32_t o = row_ptr[r - 1];
         for (int s = 0; s < m; ++s) col[o + s] = buf[s] - 1;
      }
   }
}

__global__ void to_i32(int64_t n, const int64_t* a, int32_t* b)
{
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
      b[i] = (int32_t)a[i];
}

// emap[e][a][b] = CSR index of (dof_a, dof_b) or -1.
__global__ void build_emap(int64_t ne, int nen, const int32_t* elem, const int32_t* dof,
                           const int32_t* row_ptr, const int32_t* col, int32_t* emap, int* missing)
{
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   int64_t nn2 = (int64_t)nen * nen;
   for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < ne * nn2; t += stride) {
      int64_t e = t / nn2;
      int a = (int)((t % nn2) / nen), b = (int)(t % nen);
      int32_t r = dof[elem[e * nen + a]], c = dof[elem[e * nen + b]];
      int32_t pos = -1;
      if (r && c) {
         int32_t lo = row_ptr[r - 1], hi = row_ptr[r] - 1;
         while (lo <= hi) {
            int32_t mid = (lo + hi) >> 1;
            int32_t v = col[mid];
            if (v == c - 1) { pos = mid; break; }
            if (v < c - 1) lo = mid + 1;
            else hi = mid - 1;
         }
         if (pos < 0) atomicOr(missing, 1);
      }
      emap[t] = pos;
   }
}

}  // namespace

// Equation numbers, node-to-element lists (see internal.cuh).
void finish_mesh(ofg_mesh* m)
{
   int64_t nn = m->nn, ne = m->ne;
   // equation numbers
   DBuf<int64_t> flag(nn > 0 ? nn : 1), pre(nn > 0 ? nn : 1);
   m->dof.alloc(nn > 0 ? nn : 1);
   if (nn) {
      free_flags<<<grid_for(nn, 256), 256, 0, stream()>>>(nn, m->code.p, flag.p);
      count_launch();
      scan_exclusive_i64(flag.p, pre.p, nn);
      number_dofs<<<grid_for(nn, 256), 256, 0, stream()>>>(nn, m->code.p, pre.p, m->dof.p);
      count_launch();
      OFG_LAUNCH_CHECK();
      int64_t last_pre = 0, last_flag = 0;
      OFG_CUDA(cudaMemcpyAsync(&last_pre, pre.p + nn - 1, 8, cudaMemcpyDeviceToHost, stream()));
      OFG_CUDA(cudaMemcpyAsync(&last_flag, flag.p + nn - 1, 8, cudaMemcpyDeviceToHost, stream()));
      OFG_CUDA(cudaStreamSynchronize(stream()));
      m->neq = last_pre + last_flag;
   }
   // node -> element adjacency
   DBuf<int64_t> cnt(nn + 1), start(nn + 1);
   cnt.zero();
   DBuf<int32_t> cursor(nn > 0 ? nn : 1);
   cursor.zero();
   if (ne) {
      count_n2e<<<grid_for(ne * m->nen, 256), 256, 0, stream()>>>(ne, m->nen, m->elem.p, cnt.p);
      count_launch();
   }
   scan_exclusive_i64(cnt.p, start.p, nn + 1);
   m->n2e_ptr.alloc(nn + 1);
   m->n2e.alloc(ne * m->nen > 0 ? ne * m->nen : 1);
   if (ne) {
      fill_n2e<<<grid_for(ne * m->nen, 256), 256, 0, stream()>>>(ne, m->nen, m->elem.p, start.p,
                                                                  cursor.p, m->n2e.p);
      count_launch();
   }
   finish_n2e<<<grid_for(nn + 1, 256), 256, 0, stream()>>>(nn, start.p, m->n2e_ptr.p, m->n2e.p);
   count_launch();
   OFG_LAUNCH_CHECK();

   OFG_CUDA(cudaStreamSynchronize(stream()));
}

ofg_mesh* new_mesh(int dim, int64_t nn, int64_t ne)
{
   auto m = new ofg_mesh();
   m->dim = dim;
   m->nen = dim + 1;
   m->nn = nn;
   m->ne = ne;
   m->coords.alloc(nn * dim > 0 ? nn * dim : 1);
   m->elem.alloc(ne * m->nen > 0 ? ne * m->nen : 1);
   m->code.alloc(nn > 0 ? nn : 1);
   return m;
}

}  // namespace ofg

using namespace ofg;

extern "C" {

int ofg_mesh_create_rect(double xmin, double xmax, double ymin, double ymax, int64_t nx, int64_t ny,
                         int cx0, int cxN, int cy0, int cyN, ofg_mesh** out)
{
   return guarded("ofg_mesh_create_rect", [&] {
      OFG_REQUIRE(out && nx > 0 && ny > 0, OFG_ERR_ARG, "need nx, ny > 0");
      int64_t nn = (nx + 1) * (ny + 1);
      OFG_REQUIRE(nn < (int64_t(1) << 31), OFG_ERR_SIZE, "mesh too large for int32 indices");
      ofg_mesh* m = new_mesh(2, nn, 2 * nx * ny);
      try {
         // coordinate ladders accumulated like the reference (x += hx, y += hy)
         double hx = (xmax - xmin) / (double)nx, hy = (ymax - ymin) / (double)ny;
         std::vector<double> xs(nx + 1), ys(ny + 1);
         double v = xmin;
         for (int64_t i = 0; i <= nx; ++i) { xs[i] = v; v += hx; }
         v = ymin;
         for (int64_t j = 0; j <= ny; ++j) { ys[j] = v; v += hy; }
         DBuf<double> dxs(nx + 1), dys(ny + 1);
         dxs.upload(xs.data(), nx + 1);
         dys.upload(ys.data(), ny + 1);
         rect_nodes<<<grid_for(nn, 256), 256, 0, stream()>>>(nx, ny, dxs.p, dys.p, cx0, cxN, cy0,
                                                              cyN, m->coords.p, m->code.p);
         count_launch();
         rect_elems<<<grid_for(nx * ny, 256), 256, 0, stream()>>>(nx, ny, m->elem.p);
         count_launch();
         OFG_LAUNCH_CHECK();
         finish_mesh(m);
         m->rect_nx = nx, m->rect_ny = ny;
         m->rect_code[0] = cx0, m->rect_code[1] = cxN, m->rect_code[2] = cy0, m->rect_code[3] = cyN;
      }
      catch (...) {
         delete m;
         throw;
      }
      *out = m;
   });
}

int ofg_mesh_create_kuhn(int64_t M, ofg_mesh** out)
{
   return guarded("ofg_mesh_create_kuhn", [&] {
      OFG_REQUIRE(out && M > 0, OFG_ERR_ARG, "need M > 0");
      int64_t nn = (M + 1) * (M + 1) * (M + 1), ne = 6 * M * M * M;
      OFG_REQUIRE(ne * 4 < (int64_t(1) << 31), OFG_ERR_SIZE, "mesh too large for int32 indices");
      ofg_mesh* m = new_mesh(3, nn, ne);
      try {
         kuhn_nodes<<<grid_for(nn, 256), 256, 0, stream()>>>(M, m->coords.p, m->code.p);
         count_launch();
         kuhn_elems<<<grid_for(ne, 256), 256, 0, stream()>>>(M, m->elem.p);
         count_launch();
         OFG_LAUNCH_CHECK();
         finish_mesh(m);
      }
      catch (...) {
         delete m;
         throw;
      }
      *out = m;
   });
}

int ofg_mesh_create(int dim, int64_t nn, const double* coords, int64_t ne, const int32_t* elem,
                    const int32_t* code, ofg_mesh** out)
{
   return guarded("ofg_mesh_create", [&] {
      OFG_REQUIRE(out && coords && elem && code && (dim == 2 || dim == 3) && nn > 0 && ne > 0,
                  OFG_ERR_ARG, "bad mesh arguments");
      OFG_REQUIRE(ne * (dim + 1) < (int64_t(1) << 31), OFG_ERR_SIZE, "mesh too large");
      ofg_mesh* m = new_mesh(dim, nn, ne);
      try {
         OFG_CUDA(cudaMemcpyAsync(m->coords.p, coords, nn * dim * sizeof(double), cudaMemcpyDefault,
                                  stream()));
         OFG_CUDA(cudaMemcpyAsync(m->elem.p, elem, ne * (dim + 1) * sizeof(int32_t),
                                  cudaMemcpyDefault, stream()));
         OFG_CUDA(cudaMemcpyAsync(m->code.p, code, nn * sizeof(int32_t), cudaMemcpyDefault,
                                  stream()));
         DBuf<int> bad(1);
         bad.zero();
         check_elems<<<grid_for(ne * (dim + 1), 256), 256, 0, stream()>>>(ne, dim + 1, nn,
                                                                           m->elem.p, bad.p);
         count_launch();
         OFG_LAUNCH_CHECK();
         int h = 0;
         bad.download(&h, 1);
         OFG_REQUIRE(!h, OFG_ERR_ARG, "element references a node outside [0, nn)");
         finish_mesh(m);
      }
      catch (...) {
         delete m;
         throw;
      }
      *out = m;
   });
}

int ofg_mesh_destroy(ofg_mesh* m)
{
   return guarded("ofg_mesh_destroy", [&] {
      delete m;
      OFG_CUDA(cudaStreamSynchronize(stream()));
   });
}

int ofg_mesh_info(const ofg_mesh* m, int* dim, int64_t* nn, int64_t* ne, int64_t* neq)
{
   return guarded("ofg_mesh_info", [&] {
      OFG_REQUIRE(m, OFG_ERR_ARG, "null mesh");
      if (dim) *dim = m->dim;
      if (nn) *nn = m->nn;
      if (ne) *ne = m->ne;
      if (neq) *neq = m->neq;
   });
}

int ofg_mesh_get(const ofg_mesh* m, double* coords, int32_t* elem, int32_t* code, int64_t* dof)
{
   return guarded("ofg_mesh_get", [&] {
      OFG_REQUIRE(m, OFG_ERR_ARG, "null mesh");
      if (coords)
         OFG_CUDA(cudaMemcpyAsync(coords, m->coords.p, m->nn * m->dim * sizeof(double),
                                  cudaMemcpyDefault, stream()));
      if (elem)
         OFG_CUDA(cudaMemcpyAsync(elem, m->elem.p, m->ne * m->nen * sizeof(int32_t),
                                  cudaMemcpyDefault, stream()));
      if (code)
         OFG_CUDA(cudaMemcpyAsync(code, m->code.p, m->nn * sizeof(int32_t), cudaMemcpyDefault,
                                  stream()));
      if (dof) {
         std::vector<int32_t> d = m->dof.to_host(m->nn);
         std::vector<int64_t> d64(d.begin(), d.end());
         OFG_CUDA(cudaMemcpyAsync(dof, d64.data(), m->nn * sizeof(int64_t), cudaMemcpyDefault,
                                  stream()));
      }
      OFG_CUDA(cudaStreamSynchronize(stream()));
   });
}

int ofg_mesh_set_coords(ofg_mesh* m, const double* coords)
{
   return guarded("ofg_mesh_set_coords", [&] {
      OFG_REQUIRE(m && coords, OFG_ERR_ARG, "null argument");
      OFG_CUDA(cudaMemcpyAsync(m->coords.p, coords, m->nn * m->dim * sizeof(double),
                               cudaMemcpyDefault, stream()));
      OFG_CUDA(cudaStreamSynchronize(stream()));
   });
}

int ofg_matrix_create_from_mesh(ofg_mesh* m, ofg_matrix** out)
{
   return guarded("ofg_matrix_create_from_mesh", [&] {
      OFG_REQUIRE(m && out, OFG_ERR_ARG, "null argument");
      int64_t n = m->neq, nn = m->nn;
      auto A = new ofg_matrix();
      try {
         A->n = n;
         DBuf<int64_t> len(n + 1), start(n + 1);
         len.zero();
         DBuf<int> overflow(1);
         overflow.zero();
         node_graph_rows<<<grid_for(nn, 128), 128, 0, stream()>>>(
            nn, m->nen, m->elem.p, m->dof.p, m->n2e_ptr.p, m->n2e.p, len.p, nullptr, nullptr, 0,
            overflow.p);
         count_launch();
         OFG_LAUNCH_CHECK();
         scan_exclusive_i64(len.p, start.p, n + 1);
         int64_t nnz = 0;
         int ovf = 0;
         OFG_CUDA(cudaMemcpyAsync(&nnz, start.p + n, 8, cudaMemcpyDeviceToHost, stream()));
         OFG_CUDA(cudaMemcpyAsync(&ovf, overflow.p, 4, cudaMemcpyDeviceToHost, stream()));
         OFG_CUDA(cudaStreamSynchronize(stream()));
         OFG_REQUIRE(!ovf, OFG_ERR_PATTERN, "a node touches more element DOFs than the gather limit");
         OFG_REQUIRE(nnz < (int64_t(1) << 31), OFG_ERR_PATTERN, "nnz must be below 2^31");
         A->nnz = nnz;
         A->row_ptr.alloc(n + 1);
         to_i32<<<grid_for(n + 1, 256), 256, 0, stream()>>>(n + 1, start.p, A->row_ptr.p);
         count_launch();
         A->col.alloc(nnz > 0 ? nnz : 1);
         A->val.alloc(nnz > 0 ? nnz : 1);
         A->val.zero();
         node_graph_rows<<<grid_for(nn, 128), 128, 0, stream()>>>(
            nn, m->nen, m->elem.p, m->dof.p, m->n2e_ptr.p, m->n2e.p, nullptr, A->row_ptr.p,
            A->col.p, 1, overflow.p);
         count_launch();
         OFG_LAUNCH_CHECK();
         // element -> CSR scatter map
         int64_t nmap = m->ne * m->nen * m->nen;
         A->emap.alloc(nmap > 0 ? nmap : 1);
         DBuf<int> missing(1);
         missing.zero();
         if (nmap) {
            build_emap<<<grid_for(nmap, 256), 256, 0, stream()>>>(m->ne, m->nen, m->elem.p,
                                                                   m->dof.p, A->row_ptr.p, A->col.p,
                                                                   A->emap.p, missing.p);
            count_launch();
            OFG_LAUNCH_CHECK();
         }
         int h = 0;
         missing.download(&h, 1);
         OFG_REQUIRE(!h, OFG_ERR_PATTERN, "scatter map found a pair outside the pattern");
         A->mesh = m;
         matrix_finish_pattern(A);
      }
      catch (...) {
         delete A;
         throw;
      }
      *out = A;
   });
}

}  // extern "C"
