// Headless C entry points over the reference solver (hellojxt/PPPM-TDBEM), compiled from
// the reference's own sources by oracle/Makefile into oracle/_ref/.  This file is TEST
// INFRASTRUCTURE: the parity tests, the golden-vector generator and bench.py's reference
// arm call it as the checker/baseline; the product never links it.
//
// It restates the headless part of the reference's demo driver
// (experiments/demo/main.cu:38-275: construct PPPMSolver, set_mesh / update_mesh,
// update_grid_and_face per step, read the listener cell each step) without the GL window,
// PNG dumps or the docker-based FixMesh, and adds read-out hooks for grids, histories,
// neighbour lists, cache tables and cell labels.
//
// Every entry point returns 0 on success and a nonzero code on failure (exceptions from the
// reference's launch macros, macro.h:140-167, are caught here).  Inputs are checked on the
// host against the reference's fixed list capacities (particle_grid.h:9-11,
// pppm_cache.h:79) before any reference kernel runs, because the reference itself does not
// check them without -DMEMORY_CHECK.
#include <cstdint>
#include <cstring>
#include <map>
#include <set>
#include <stdexcept>
#include <unordered_set>
#include <vector>
#include "ghost_cell.h"
#include "ghost_cell_util.h"
#include "pppm.h"
#include "pppm_direct.h"

using namespace pppm;

namespace
{

enum
{
    REF_OK = 0,
    REF_ERR_ARG = 1,
    REF_ERR_CUDA = 2,
    REF_ERR_CAPACITY = 3,
    REF_ERR_STATE = 5,
};

// Host-side check that a mesh keeps every reference list inside its capacity with margin
// and keeps every triangle away from the grid edge (the reference reads cells up to two
// layers away from a triangle's cell without bounds checks).
struct CapacityCheck
{
    int res;
    float dl;
    float3 min_pos;
    std::vector<std::unordered_set<int>> seen_pairs;  // distinct face-cache pairs per centre

    int check(const float *V, int nv, const int *F, int nt, bool track_pairs)
    {
        std::vector<int> cell_of(nt), base_of(nt);
        std::vector<int> count((size_t)res * res * res, 0), bcount((size_t)res * res * res, 0);
        for (int i = 0; i < nt; i++)
        {
            int a = F[3 * i], b = F[3 * i + 1], c = F[3 * i + 2];
            if (a < 0 || b < 0 || c < 0 || a >= nv || b >= nv || c >= nv)
                return REF_ERR_ARG;
            float cx = (V[3 * a] + V[3 * b] + V[3 * c]) / 3.0f;
            float cy = (V[3 * a + 1] + V[3 * b + 1] + V[3 * c + 1]) / 3.0f;
            float cz = (V[3 * a + 2] + V[3 * b + 2] + V[3 * c + 2]) / 3.0f;
            float p[3] = {(cx - min_pos.x) / dl, (cy - min_pos.y) / dl, (cz - min_pos.z) / dl};
            int q[3], bq[3];
            for (int d = 0; d < 3; d++)
            {
                q[d] = (int)p[d];
                bq[d] = q[d] - ((p[d] - (q[d] + 0.5f)) < 0 ? 1 : 0);
                if (q[d] < 3 || q[d] > res - 4 || bq[d] < 3 || bq[d] > res - 4)
                    return REF_ERR_CAPACITY;
            }
            cell_of[i] = (q[0] * res + q[1]) * res + q[2];
            base_of[i] = (bq[0] * res + bq[1]) * res + bq[2];
            count[cell_of[i]]++;
            bcount[base_of[i]]++;
        }
        for (size_t c = 0; c < count.size(); c++)
            if (count[c] > 100 || bcount[c] > 100)
                return REF_ERR_CAPACITY;
        auto block_sum = [&](int cell, int lo, int hi) {
            int x = cell / (res * res), y = (cell / res) % res, z = cell % res, s = 0;
            for (int dx = lo; dx <= hi; dx++)
                for (int dy = lo; dy <= hi; dy++)
                    for (int dz = lo; dz <= hi; dz++)
                        s += count[((x + dx) * res + (y + dy)) * res + (z + dz)];
            return s;
        };
        for (int i = 0; i < nt; i++)
        {
            // every cell whose 3^3 block holds triangle i lies within one cell of it
            int x = cell_of[i] / (res * res), y = (cell_of[i] / res) % res, z = cell_of[i] % res;
            for (int dx = -1; dx <= 1; dx++)
                for (int dy = -1; dy <= 1; dy++)
                    for (int dz = -1; dz <= 1; dz++)
                        if (block_sum(((x + dx) * res + (y + dy)) * res + (z + dz), -1, 1) > 230)
                            return REF_ERR_CAPACITY;
            if (block_sum(base_of[i], -1, 2) > 460)
                return REF_ERR_CAPACITY;
        }
        if (track_pairs)
        {
            if ((int)seen_pairs.size() != nt)
                seen_pairs.assign(nt, {});
            std::map<int, std::vector<int>> by_cell;
            for (int i = 0; i < nt; i++)
                by_cell[cell_of[i]].push_back(i);
            for (int i = 0; i < nt; i++)
            {
                int b = base_of[i];
                int x = b / (res * res), y = (b / res) % res, z = b % res;
                for (int dx = -1; dx <= 2; dx++)
                    for (int dy = -1; dy <= 2; dy++)
                        for (int dz = -1; dz <= 2; dz++)
                        {
                            auto it = by_cell.find(((x + dx) * res + (y + dy)) * res + (z + dz));
                            if (it != by_cell.end())
                                for (int j : it->second)
                                    seen_pairs[i].insert(j);
                        }
                if (seen_pairs[i].size() > 1000)
                    return REF_ERR_CAPACITY;
            }
        }
        return REF_OK;
    }
};

struct RefPPPM
{
    PPPMSolver *solver = nullptr;
    CapacityCheck cap;
    bool checks = true;
    int nv = 0, nt = 0;
    std::vector<float> verts;
    GArr<float> acc_dev;
};

struct RefCells
{
    GhostCellSolver *solver = nullptr;
    CapacityCheck cap;
    int nv = 0, nt = 0;
};

template <typename F>
int guarded(F &&f)
{
    try
    {
        return f();
    }
    catch (const std::exception &e)
    {
        fprintf(stderr, "[pppm_ref] %s\n", e.what());
        return REF_ERR_CUDA;
    }
}

int last_cuda_status()
{
    cudaError_t e = cudaDeviceSynchronize();
    if (e == cudaSuccess)
        e = cudaGetLastError();
    return e == cudaSuccess ? REF_OK : REF_ERR_CUDA;
}

CArr<float3> to_float3(const float *V, int nv)
{
    CArr<float3> out(nv);
    for (int i = 0; i < nv; i++)
        out[i] = make_float3(V[3 * i], V[3 * i + 1], V[3 * i + 2]);
    return out;
}

CArr<int3> to_int3(const int *F, int nt)
{
    CArr<int3> out(nt);
    for (int i = 0; i < nt; i++)
        out[i] = make_int3(F[3 * i], F[3 * i + 1], F[3 * i + 2]);
    return out;
}

__global__ void gather_face_weights_kernel(FaceCache fc, const int *centre, const int *nbr, int n, LayerWeightHalf *out)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    int slot = fc.cache_index(centre[i], nbr[i]);
    if (slot < 0)
    {
        memset(&out[i], 0, sizeof(LayerWeightHalf));
        return;
    }
    out[i] = fc.cache(centre[i], slot).weight;
}

__global__ void laplace_weight_kernel(TDBEM bem, const float3 *verts, int3 src, int3 dst_face, float3 dst_point,
                                      int to_point, float *out)
{
    LayerWeight<float> w;
    if (to_point)
        bem.laplace_weight(verts, PairInfo(src, dst_point), &w);
    else
        bem.laplace_weight(verts, PairInfo(src, dst_face), &w);
    for (int k = 0; k < STEP_NUM; k++)
    {
        out[k] = w.single_layer[k];
        out[STEP_NUM + k] = w.double_layer[k];
    }
}

__global__ void laplace_weight_complex_kernel(TDBEM bem, const float3 *verts, int3 src, int3 dst_face,
                                              float3 dst_point, int to_point, float *out)
{
    LayerWeight<cpx> w;
    if (to_point)
        bem.laplace_weight(verts, PairInfo(src, dst_point), &w);
    else
        bem.laplace_weight(verts, PairInfo(src, dst_face), &w);
    for (int k = 0; k < STEP_NUM; k++)
    {
        out[4 * k + 0] = w.single_layer[k].real();
        out[4 * k + 1] = w.single_layer[k].imag();
        out[4 * k + 2] = w.double_layer[k].real();
        out[4 * k + 3] = w.double_layer[k].imag();
    }
}

__global__ void read_history_kernel(GArr<History> neumann, GArr<History> dirichlet, float *n_out, float *d_out)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= neumann.size())
        return;
    for (int k = 0; k < STEP_NUM * 2; k++)
    {
        n_out[i * STEP_NUM * 2 + k] = neumann[i][k];
        d_out[i * STEP_NUM * 2 + k] = dirichlet[i][k];
    }
}

__global__ void write_history_kernel(GArr<History> neumann, GArr<History> dirichlet, const float *n_in,
                                     const float *d_in)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= neumann.size())
        return;
    for (int k = 0; k < STEP_NUM * 2; k++)
    {
        neumann[i][k] = n_in[i * STEP_NUM * 2 + k];
        dirichlet[i][k] = d_in[i * STEP_NUM * 2 + k];
    }
}

}  // namespace

extern "C" {

int ref_abi_version() { return 1; }

// ---------------------------------------------------------------- PPPMSolver -----------
void *ref_pppm_create(int res, float dl, float dt, const float *min_pos, float reflect_coeff)
{
    if (res < 8 || dl <= 0 || dt <= 0)
        return nullptr;
    RefPPPM *h = new RefPPPM();
    try
    {
        h->solver = new PPPMSolver(res, dl, dt, make_float3(min_pos[0], min_pos[1], min_pos[2]), 0, reflect_coeff);
    }
    catch (const std::exception &e)
    {
        fprintf(stderr, "[pppm_ref] %s\n", e.what());
        delete h;
        return nullptr;
    }
    h->cap.res = res;
    h->cap.dl = dl;
    h->cap.min_pos = make_float3(min_pos[0], min_pos[1], min_pos[2]);
    return h;
}

void ref_pppm_destroy(void *p)
{
    RefPPPM *h = (RefPPPM *)p;
    if (!h)
        return;
    if (h->solver)
    {
        h->solver->clear();
        delete h->solver;
    }
    h->acc_dev.clear();
    delete h;
}

int ref_pppm_set_mesh(void *p, const float *V, int nv, const int *F, int nt)
{
    RefPPPM *h = (RefPPPM *)p;
    if (!h || nv <= 0 || nt <= 0 || h->solver->mesh_set)
        return REF_ERR_ARG;
    int rc = h->cap.check(V, nv, F, nt, true);
    if (rc)
        return rc;
    h->nv = nv;
    h->nt = nt;
    return guarded([&] {
        CArr<float3> verts = to_float3(V, nv);
        CArr<int3> tris = to_int3(F, nt);
        h->solver->set_mesh(verts, tris);
        h->acc_dev.resize(nt);
        return last_cuda_status();
    });
}

int ref_pppm_update_mesh(void *p, const float *V)
{
    RefPPPM *h = (RefPPPM *)p;
    if (!h || !h->solver->mesh_set)
        return REF_ERR_STATE;
    auto tris = h->solver->pg.faces.cpu();
    std::vector<int> F(3 * h->nt);
    for (int i = 0; i < h->nt; i++)
    {
        F[3 * i] = tris[i].x;
        F[3 * i + 1] = tris[i].y;
        F[3 * i + 2] = tris[i].z;
    }
    if (h->checks)
    {
        int rc = h->cap.check(V, h->nv, F.data(), h->nt, true);
        if (rc)
            return rc;
    }
    return guarded([&] {
        CArr<float3> verts = to_float3(V, h->nv);
        h->solver->update_mesh(verts);
        return last_cuda_status();
    });
}

// Host-only capacity check of a vertex set against this solver's topology (no reference
// code runs); used to validate a whole trajectory before timing it with checks disabled.
int ref_pppm_check_mesh(void *p, const float *V)
{
    RefPPPM *h = (RefPPPM *)p;
    if (!h || !h->solver->mesh_set)
        return REF_ERR_STATE;
    auto tris = h->solver->pg.faces.cpu();
    std::vector<int> F(3 * h->nt);
    for (int i = 0; i < h->nt; i++)
    {
        F[3 * i] = tris[i].x;
        F[3 * i + 1] = tris[i].y;
        F[3 * i + 2] = tris[i].z;
    }
    return h->cap.check(V, h->nv, F.data(), h->nt, true);
}

// Enable (default) or disable the per-update host capacity check.
int ref_pppm_set_checks(void *p, int on)
{
    RefPPPM *h = (RefPPPM *)p;
    if (!h)
        return REF_ERR_ARG;
    h->checks = on != 0;
    return REF_OK;
}

// One reference step per row of acc (host array, nsteps x nt).  After each step the
// listener cells are read exactly as the demo driver does (experiments/demo/main.cu:266):
// grids[t](x, y, z) copied to the host.  out: nsteps x nlisten.
int ref_pppm_run(void *p, const float *acc, int nsteps, const int *listen_xyz, int nlisten, float *out)
{
    RefPPPM *h = (RefPPPM *)p;
    if (!h || !h->solver->mesh_set || nsteps < 0)
        return REF_ERR_STATE;
    int res = h->solver->res();
    for (int l = 0; l < nlisten; l++)
        for (int d = 0; d < 3; d++)
            if (listen_xyz[3 * l + d] < 0 || listen_xyz[3 * l + d] >= res)
                return REF_ERR_ARG;
    return guarded([&] {
        CArr<float> row(h->nt);
        for (int s = 0; s < nsteps; s++)
        {
            memcpy(row.data(), acc + (size_t)s * h->nt, sizeof(float) * h->nt);
            h->solver->update_grid_and_face(row);
            for (int l = 0; l < nlisten; l++)
                out[(size_t)s * nlisten + l] =
                    h->solver->pg.fdtd.grids[h->solver->pg.fdtd.t](
                        to_cpu(listen_xyz[3 * l], listen_xyz[3 * l + 1], listen_xyz[3 * l + 2]));
        }
        return last_cuda_status();
    });
}

// Same as ref_pppm_run but with device-resident accelerations (one upload per step from a
// device pointer), used for timing the reference path without host-side copies per step.
int ref_pppm_run_device(void *p, const float *acc_dev, int nsteps, int listen_x, int listen_y, int listen_z,
                        float *out)
{
    RefPPPM *h = (RefPPPM *)p;
    if (!h || !h->solver->mesh_set || nsteps < 0)
        return REF_ERR_STATE;
    return guarded([&] {
        for (int s = 0; s < nsteps; s++)
        {
            GArr<float> row((float *)(acc_dev + (size_t)s * h->nt), h->nt);
            h->solver->update_grid_and_face(row);
            if (out)
                out[s] = h->solver->pg.fdtd.grids[h->solver->pg.fdtd.t](to_cpu(listen_x, listen_y, listen_z));
        }
        return last_cuda_status();
    });
}

int ref_pppm_time(void *p)
{
    RefPPPM *h = (RefPPPM *)p;
    return h ? h->solver->pg.fdtd.t : -1000;
}

// Grid slot t + rel (rel in {0,-1,-2}); res^3 floats, x-major, z contiguous.
int ref_pppm_read_grid(void *p, int rel, float *out)
{
    RefPPPM *h = (RefPPPM *)p;
    if (!h || rel > 0 || rel < -2)
        return REF_ERR_ARG;
    auto &g = h->solver->pg.fdtd.grids[h->solver->pg.fdtd.t + rel];
    return guarded([&] {
        cudaMemcpy(out, g.data.data(), sizeof(float) * g.data.size(), cudaMemcpyDeviceToHost);
        return last_cuda_status();
    });
}

int ref_pppm_write_grid(void *p, int rel, const float *in)
{
    RefPPPM *h = (RefPPPM *)p;
    if (!h || rel > 0 || rel < -2)
        return REF_ERR_ARG;
    auto &g = h->solver->pg.fdtd.grids[h->solver->pg.fdtd.t + rel];
    return guarded([&] {
        cudaMemcpy(g.data.data(), in, sizeof(float) * g.data.size(), cudaMemcpyHostToDevice);
        return last_cuda_status();
    });
}

int ref_pppm_read_far(void *p, float *out)
{
    RefPPPM *h = (RefPPPM *)p;
    if (!h)
        return REF_ERR_ARG;
    auto &g = h->solver->grid_far_field[h->solver->pg.fdtd.t];
    return guarded([&] {
        cudaMemcpy(out, g.data.data(), sizeof(float) * g.data.size(), cudaMemcpyDeviceToHost);
        return last_cuda_status();
    });
}

// Histories as stored: nt x 32 ring slots each (slot = time mod 32).
int ref_pppm_read_history(void *p, float *neumann, float *dirichlet)
{
    RefPPPM *h = (RefPPPM *)p;
    if (!h || !h->solver->mesh_set)
        return REF_ERR_STATE;
    return guarded([&] {
        float *dn, *dd;
        size_t bytes = sizeof(float) * h->nt * STEP_NUM * 2;
        cudaMalloc(&dn, bytes);
        cudaMalloc(&dd, bytes);
        read_history_kernel<<<(h->nt + 63) / 64, 64>>>(h->solver->neumann, h->solver->dirichlet, dn, dd);
        cudaMemcpy(neumann, dn, bytes, cudaMemcpyDeviceToHost);
        cudaMemcpy(dirichlet, dd, bytes, cudaMemcpyDeviceToHost);
        cudaFree(dn);
        cudaFree(dd);
        return last_cuda_status();
    });
}

int ref_pppm_write_history(void *p, const float *neumann, const float *dirichlet)
{
    RefPPPM *h = (RefPPPM *)p;
    if (!h || !h->solver->mesh_set)
        return REF_ERR_STATE;
    return guarded([&] {
        float *dn, *dd;
        size_t bytes = sizeof(float) * h->nt * STEP_NUM * 2;
        cudaMalloc(&dn, bytes);
        cudaMalloc(&dd, bytes);
        cudaMemcpy(dn, neumann, bytes, cudaMemcpyHostToDevice);
        cudaMemcpy(dd, dirichlet, bytes, cudaMemcpyHostToDevice);
        write_history_kernel<<<(h->nt + 63) / 64, 64>>>(h->solver->neumann, h->solver->dirichlet, dn, dd);
        cudaDeviceSynchronize();
        cudaFree(dn);
        cudaFree(dd);
        return last_cuda_status();
    });
}

// Triangle records: geom nt x 7 (center xyz, normal xyz, area), cells nt x 6 (grid coord,
// base coord).
int ref_pppm_read_triangles(void *p, float *geom, int *cells)
{
    RefPPPM *h = (RefPPPM *)p;
    if (!h || !h->solver->mesh_set)
        return REF_ERR_STATE;
    return guarded([&] {
        auto tris = h->solver->pg.triangles.cpu();
        for (int i = 0; i < h->nt; i++)
        {
            const Triangle &t = tris[i];
            float g[7] = {t.center.x, t.center.y, t.center.z, t.normal.x, t.normal.y, t.normal.z, t.area};
            int c[6] = {t.grid_coord.x,      t.grid_coord.y,      t.grid_coord.z,
                        t.grid_base_coord.x, t.grid_base_coord.y, t.grid_base_coord.z};
            memcpy(geom + 7 * i, g, sizeof(g));
            memcpy(cells + 6 * i, c, sizeof(c));
        }
        return last_cuda_status();
    });
}

// Sizes of the neighbour structures: n3 = non-empty 3^3 cells, p3 = total 3^3 list entries,
// b4 = non-empty base cells, p4 = total 4^3 list entries summed over base cells.
int ref_pppm_list_sizes(void *p, int *sizes)
{
    RefPPPM *h = (RefPPPM *)p;
    if (!h || !h->solver->mesh_set)
        return REF_ERR_STATE;
    return guarded([&] {
        auto &pg = h->solver->pg;
        auto n3 = pg.neighbor_3_square_nonempty.data.cpu();
        auto b4 = pg.base_coord_nonempty.data.cpu();
        int n3n = pg.neighbor_3_square_nonempty.size(), b4n = pg.base_coord_nonempty.size();
        long p3 = 0, p4 = 0;
        auto l3 = pg.neighbor_3_square_list.cpu();
        auto l4 = pg.neighbor_4_square_list.cpu();
        for (int i = 0; i < n3n; i++)
            p3 += l3(n3[i].coord).size();
        for (int i = 0; i < b4n; i++)
            p4 += l4(b4[i].coord).size();
        sizes[0] = n3n;
        sizes[1] = (int)p3;
        sizes[2] = b4n;
        sizes[3] = (int)p4;
        return last_cuda_status();
    });
}

// n3_cells: n3 x 4 (x, y, z, list length) in the reference's compacted order;
// p3_tris: concatenated 3^3 lists (reference order, which is atomic-append order inside a cell);
// b4_cells: b4 x 4 (x, y, z, base-list length); b4_lists: concatenated base-cell face lists;
// p4_tris: concatenated 4^3 lists; cell_counts: res^3 per-cell face counts.
int ref_pppm_read_lists(void *p, int *n3_cells, int *p3_tris, int *b4_cells, int *b4_lists, int *p4_tris,
                        int *cell_counts)
{
    RefPPPM *h = (RefPPPM *)p;
    if (!h || !h->solver->mesh_set)
        return REF_ERR_STATE;
    return guarded([&] {
        auto &pg = h->solver->pg;
        auto n3 = pg.neighbor_3_square_nonempty.data.cpu();
        auto b4 = pg.base_coord_nonempty.data.cpu();
        int n3n = pg.neighbor_3_square_nonempty.size(), b4n = pg.base_coord_nonempty.size();
        auto l3 = pg.neighbor_3_square_list.cpu();
        auto l4 = pg.neighbor_4_square_list.cpu();
        auto bl = pg.base_coord_face_list.cpu();
        auto gl = pg.grid_face_list.cpu();
        long o3 = 0, o4 = 0, ob = 0;
        for (int i = 0; i < n3n; i++)
        {
            auto &lst = l3(n3[i].coord);
            int c[4] = {n3[i].coord.x, n3[i].coord.y, n3[i].coord.z, lst.size()};
            memcpy(n3_cells + 4 * i, c, sizeof(c));
            for (int j = 0; j < lst.size(); j++)
                p3_tris[o3++] = lst.list[j];
        }
        for (int i = 0; i < b4n; i++)
        {
            auto &lst = l4(b4[i].coord);
            auto &base = bl(b4[i].coord);
            int c[4] = {b4[i].coord.x, b4[i].coord.y, b4[i].coord.z, base.size()};
            memcpy(b4_cells + 4 * i, c, sizeof(c));
            for (int j = 0; j < base.size(); j++)
                b4_lists[ob++] = base.list[j];
            for (int j = 0; j < lst.size(); j++)
                p4_tris[o4++] = lst.list[j];
        }
        int res = h->solver->res();
        for (int x = 0; x < res; x++)
            for (int y = 0; y < res; y++)
                for (int z = 0; z < res; z++)
                    cell_counts[(x * res + y) * res + z] = gl(x, y, z).size();
        return last_cuda_status();
    });
}

// GridCache weights: nt x 54 LayerWeightHalf records (27 FDTD-near then 27 BEM-near), each
// 72 bytes: 16 half single-layer, float scale, 16 half double-layer, float scale
// (bem.h:163-169, pppm_cache.h:13-20).
int ref_pppm_read_grid_cache(void *p, void *out)
{
    RefPPPM *h = (RefPPPM *)p;
    if (!h || !h->solver->mesh_set)
        return REF_ERR_STATE;
    static_assert(sizeof(LayerWeightHalf) == 72, "LayerWeightHalf layout");
    return guarded([&] {
        auto cache = h->solver->grid_cache.cache.cpu();
        char *dst = (char *)out;
        for (int i = 0; i < h->nt; i++)
        {
            memcpy(dst, cache[i].fdtd_near_weight, 27 * sizeof(LayerWeightHalf));
            dst += 27 * sizeof(LayerWeightHalf);
            memcpy(dst, cache[i].bem_near_weight, 27 * sizeof(LayerWeightHalf));
            dst += 27 * sizeof(LayerWeightHalf);
        }
        return last_cuda_status();
    });
}

// FaceCache weights for explicit (centre, neighbour) pairs; pairs that were never cached
// come back zero-filled.
int ref_pppm_read_face_cache(void *p, const int *centre, const int *nbr, int n, void *out)
{
    RefPPPM *h = (RefPPPM *)p;
    if (!h || !h->solver->mesh_set || n < 0)
        return REF_ERR_STATE;
    for (int i = 0; i < n; i++)
        if (centre[i] < 0 || centre[i] >= h->nt || nbr[i] < 0 || nbr[i] >= h->nt)
            return REF_ERR_ARG;
    if (n == 0)
        return REF_OK;
    return guarded([&] {
        int *dc, *dn;
        LayerWeightHalf *dw;
        cudaMalloc(&dc, sizeof(int) * n);
        cudaMalloc(&dn, sizeof(int) * n);
        cudaMalloc(&dw, sizeof(LayerWeightHalf) * n);
        cudaMemcpy(dc, centre, sizeof(int) * n, cudaMemcpyHostToDevice);
        cudaMemcpy(dn, nbr, sizeof(int) * n, cudaMemcpyHostToDevice);
        gather_face_weights_kernel<<<(n + 127) / 128, 128>>>(h->solver->face_cache, dc, dn, n, dw);
        cudaMemcpy(out, dw, sizeof(LayerWeightHalf) * n, cudaMemcpyDeviceToHost);
        cudaFree(dc);
        cudaFree(dn);
        cudaFree(dw);
        return last_cuda_status();
    });
}

int ref_pppm_read_interp(void *p, float *out)
{
    RefPPPM *h = (RefPPPM *)p;
    if (!h || !h->solver->mesh_set)
        return REF_ERR_STATE;
    return guarded([&] {
        auto w = h->solver->face_cache.interpolation_weight.cpu();
        memcpy(out, w.begin(), sizeof(float) * 8 * h->nt);
        return last_cuda_status();
    });
}

// The reference's own uncached evaluation (pppm.cu:227-240, pppm_direct.cu): one FDTD step
// followed by the direct far/near correction.  Used by the GridCache known-answer check
// (tests/GridCacheTest.cu:16-64).
int ref_pppm_direct_step(void *p)
{
    RefPPPM *h = (RefPPPM *)p;
    if (!h || !h->solver->mesh_set)
        return REF_ERR_STATE;
    return guarded([&] {
        h->solver->solve_fdtd_far_simple();
        h->solver->solve_fdtd_near_simple();
        return last_cuda_status();
    });
}

int ref_pppm_cached_correction_step(void *p)
{
    RefPPPM *h = (RefPPPM *)p;
    if (!h || !h->solver->mesh_set)
        return REF_ERR_STATE;
    return guarded([&] {
        h->solver->pg.fdtd.step();
        h->solver->solve_fdtd_far();
        h->solver->solve_fdtd_near();
        return last_cuda_status();
    });
}

int ref_pppm_reset_fields(void *p)
{
    RefPPPM *h = (RefPPPM *)p;
    if (!h)
        return REF_ERR_ARG;
    return guarded([&] {
        h->solver->pg.fdtd.reset();
        if (h->solver->mesh_set)
        {
            h->solver->neumann.reset();
            h->solver->dirichlet.reset();
        }
        return last_cuda_status();
    });
}

// Single TDBEM weight on the device with the reference's arithmetic (bem.h:306-351):
// out[0:16] single layer, out[16:32] double layer.
int ref_laplace_weight(float dt, float dl, const float *V, int nv, const int *src, int to_point, const int *dst_face,
                       const float *dst_point, float *out)
{
    return guarded([&] {
        TDBEM bem;
        bem.init(dt, dl);
        float3 *dv;
        float *dout;
        cudaMalloc(&dv, sizeof(float3) * nv);
        cudaMalloc(&dout, sizeof(float) * 2 * STEP_NUM);
        cudaMemcpy(dv, V, sizeof(float3) * nv, cudaMemcpyHostToDevice);
        int3 s = make_int3(src[0], src[1], src[2]);
        int3 df = to_point ? make_int3(0, 0, 0) : make_int3(dst_face[0], dst_face[1], dst_face[2]);
        float3 dp = to_point ? make_float3(dst_point[0], dst_point[1], dst_point[2]) : make_float3(0, 0, 0);
        laplace_weight_kernel<<<1, 1>>>(bem, dv, s, df, dp, to_point, dout);
        cudaMemcpy(out, dout, sizeof(float) * 2 * STEP_NUM, cudaMemcpyDeviceToHost);
        cudaFree(dv);
        cudaFree(dout);
        return last_cuda_status();
    });
}

// Same pair, Laplace-domain values before the FFT (k <= 8 evaluated, k > 8 conjugates):
// out is 16 x (re_single, im_single, re_double, im_double).
int ref_laplace_spectrum(float dt, float dl, const float *V, int nv, const int *src, int to_point, const int *dst_face,
                         const float *dst_point, float *out)
{
    return guarded([&] {
        TDBEM bem;
        bem.init(dt, dl);
        float3 *dv;
        float *dout;
        cudaMalloc(&dv, sizeof(float3) * nv);
        cudaMalloc(&dout, sizeof(float) * 4 * STEP_NUM);
        cudaMemcpy(dv, V, sizeof(float3) * nv, cudaMemcpyHostToDevice);
        int3 s = make_int3(src[0], src[1], src[2]);
        int3 df = to_point ? make_int3(0, 0, 0) : make_int3(dst_face[0], dst_face[1], dst_face[2]);
        float3 dp = to_point ? make_float3(dst_point[0], dst_point[1], dst_point[2]) : make_float3(0, 0, 0);
        laplace_weight_complex_kernel<<<1, 1>>>(bem, dv, s, df, dp, to_point, dout);
        cudaMemcpy(out, dout, sizeof(float) * 4 * STEP_NUM, cudaMemcpyDeviceToHost);
        cudaFree(dv);
        cudaFree(dout);
        return last_cuda_status();
    });
}

// TDBEM::init on the host (bem.h:264-277): lambda and the 16 wave numbers (re, im).
int ref_tdbem_init(float dt, float dl, float *lambda, float *wave_numbers)
{
    TDBEM bem;
    bem.init(dt, dl);
    *lambda = bem.lambda;
    for (int k = 0; k < STEP_NUM; k++)
    {
        wave_numbers[2 * k] = bem.wave_numbers[k].real();
        wave_numbers[2 * k + 1] = bem.wave_numbers[k].imag();
    }
    return REF_OK;
}

// ---------------------------------------------------------------- bare FDTD ------------
void *ref_fdtd_create(int res, float dl, float dt, int pml_width)
{
    if (res < 8)
        return nullptr;
    FDTD *f = new FDTD();
    try
    {
        f->init(res, dl, dt, pml_width);
    }
    catch (const std::exception &e)
    {
        fprintf(stderr, "[pppm_ref] %s\n", e.what());
        delete f;
        return nullptr;
    }
    return f;
}

void ref_fdtd_destroy(void *p)
{
    FDTD *f = (FDTD *)p;
    if (!f)
        return;
    f->clear();
    delete f;
}

int ref_fdtd_step(void *p, int n)
{
    FDTD *f = (FDTD *)p;
    if (!f || n < 0)
        return REF_ERR_ARG;
    return guarded([&] {
        for (int i = 0; i < n; i++)
            f->step();
        return last_cuda_status();
    });
}

int ref_fdtd_time(void *p) { return p ? ((FDTD *)p)->t : -1000; }

int ref_fdtd_read(void *p, int rel, float *out)
{
    FDTD *f = (FDTD *)p;
    if (!f || rel > 0 || rel < -2)
        return REF_ERR_ARG;
    auto &g = f->grids[f->t + rel];
    return guarded([&] {
        cudaMemcpy(out, g.data.data(), sizeof(float) * g.data.size(), cudaMemcpyDeviceToHost);
        return last_cuda_status();
    });
}

int ref_fdtd_write(void *p, int rel, const float *in)
{
    FDTD *f = (FDTD *)p;
    if (!f || rel > 0 || rel < -2)
        return REF_ERR_ARG;
    auto &g = f->grids[f->t + rel];
    return guarded([&] {
        cudaMemcpy(g.data.data(), in, sizeof(float) * g.data.size(), cudaMemcpyHostToDevice);
        return last_cuda_status();
    });
}

// PML auxiliary fields of slot t + rel: res^3 x 6 floats (v1 xyz, v2 xyz), fdtd.h:12-16.
int ref_fdtd_read_pml(void *p, int rel, float *out)
{
    FDTD *f = (FDTD *)p;
    if (!f || rel > 0 || rel < -2)
        return REF_ERR_ARG;
    auto &g = f->pml_grids[f->t + rel];
    return guarded([&] {
        cudaMemcpy(out, g.data.data(), sizeof(PMLCell) * g.data.size(), cudaMemcpyDeviceToHost);
        return last_cuda_status();
    });
}

// ---------------------------------------------------------------- cell labels ----------
// Cell classification and fresh-cell fill of the ghost-cell solver
// (ghost_cell_util.cu:7-230, ghost_cell.cu:51-218), driven without the ghost-cell linear
// system: set_mesh/update_mesh below run only the particle grid, fill_cell_data and
// fill_in_fresh_cell.
void *ref_cells_create(int res, float dl, float dt, const float *min_pos)
{
    if (res < 8)
        return nullptr;
    RefCells *h = new RefCells();
    try
    {
        h->solver = new GhostCellSolver(make_float3(min_pos[0], min_pos[1], min_pos[2]), dl, res, dt);
    }
    catch (const std::exception &e)
    {
        fprintf(stderr, "[pppm_ref] %s\n", e.what());
        delete h;
        return nullptr;
    }
    h->cap.res = res;
    h->cap.dl = dl;
    h->cap.min_pos = make_float3(min_pos[0], min_pos[1], min_pos[2]);
    return h;
}

void ref_cells_destroy(void *p)
{
    RefCells *h = (RefCells *)p;
    if (!h)
        return;
    if (h->solver)
    {
        h->solver->fresh_cell_list.clear();
        h->solver->cell_data.clear();
        h->solver->cell_data_old.clear();
        h->solver->grid.clear();
        h->solver->neuuman_data.clear();
        h->solver->neuuman_data_old.clear();
        h->solver->fresh_error.clear();
        delete h->solver;
    }
    delete h;
}

int ref_cells_set_mesh(void *p, const float *V, int nv, const int *F, int nt, const float *acc)
{
    RefCells *h = (RefCells *)p;
    if (!h || nv <= 0 || nt <= 0)
        return REF_ERR_ARG;
    int rc = h->cap.check(V, nv, F, nt, false);
    if (rc)
        return rc;
    h->nv = nv;
    h->nt = nt;
    return guarded([&] {
        auto &s = *h->solver;
        CArr<float3> verts = to_float3(V, nv);
        CArr<int3> tris = to_int3(F, nt);
        s.grid.set_mesh(verts, tris);
        s.ghost_cell_num = fill_cell_data(s.grid, s.cell_data, false);
        CArr<float> a(nt);
        for (int i = 0; i < nt; i++)
            a[i] = acc ? acc[i] : 0.0f;
        s.neuuman_data.assign(a);
        s.neuuman_data_old.assign(a);
        return last_cuda_status();
    });
}

// Move the mesh, re-label, and fill fresh cells in grids[t] and grids[t-1] of the solver's
// own FDTD grid.  acc: the new per-triangle accelerations (the previous ones become "old").
int ref_cells_update_mesh(void *p, const float *V, const float *acc)
{
    RefCells *h = (RefCells *)p;
    if (!h || h->nt == 0)
        return REF_ERR_STATE;
    auto faces = h->solver->grid.faces.cpu();
    std::vector<int> F(3 * h->nt);
    for (int i = 0; i < h->nt; i++)
    {
        F[3 * i] = faces[i].x;
        F[3 * i + 1] = faces[i].y;
        F[3 * i + 2] = faces[i].z;
    }
    int rc = h->cap.check(V, h->nv, F.data(), h->nt, false);
    if (rc)
        return rc;
    return guarded([&] {
        auto &s = *h->solver;
        CArr<float3> verts = to_float3(V, h->nv);
        s.grid.update_mesh(verts);
        s.cell_data_old.assign(s.cell_data);
        s.ghost_cell_num = fill_cell_data(s.grid, s.cell_data, false);
        CArr<float> a(h->nt);
        for (int i = 0; i < h->nt; i++)
            a[i] = acc ? acc[i] : 0.0f;
        s.neuuman_data_old.assign(s.neuuman_data);
        s.neuuman_data.assign(a);
        s.fill_in_fresh_cell();
        return last_cuda_status();
    });
}

// Per-cell records, res^3 each: type (AIR 0, SOLID 1, GHOST 2, UNKNOWN 3), nearest triangle,
// ghost index; point data res^3 x 3 (nearest point, reflect point); distance res^3.
int ref_cells_read(void *p, int *type, int *nearest, int *ghost_idx, float *nearest_point, float *reflect_point,
                   float *dist)
{
    RefCells *h = (RefCells *)p;
    if (!h)
        return REF_ERR_ARG;
    return guarded([&] {
        auto cells = h->solver->cell_data.cpu();
        int n = h->solver->res();
        size_t total = (size_t)n * n * n;
        for (size_t i = 0; i < total; i++)
        {
            const CellInfo &c = cells.data[i];
            type[i] = (int)c.type;
            nearest[i] = c.nearest_particle_idx;
            ghost_idx[i] = c.ghost_idx;
            nearest_point[3 * i] = c.nearst_point.x;
            nearest_point[3 * i + 1] = c.nearst_point.y;
            nearest_point[3 * i + 2] = c.nearst_point.z;
            reflect_point[3 * i] = c.reflect_point.x;
            reflect_point[3 * i + 1] = c.reflect_point.y;
            reflect_point[3 * i + 2] = c.reflect_point.z;
            dist[i] = c.nearst_distance;
        }
        return last_cuda_status();
    });
}

int ref_cells_write_grid(void *p, int rel, const float *in)
{
    RefCells *h = (RefCells *)p;
    if (!h || rel > 0 || rel < -2)
        return REF_ERR_ARG;
    auto &f = h->solver->grid.fdtd;
    auto &g = f.grids[f.t + rel];
    return guarded([&] {
        cudaMemcpy(g.data.data(), in, sizeof(float) * g.data.size(), cudaMemcpyHostToDevice);
        return last_cuda_status();
    });
}

int ref_cells_read_grid(void *p, int rel, float *out)
{
    RefCells *h = (RefCells *)p;
    if (!h || rel > 0 || rel < -2)
        return REF_ERR_ARG;
    auto &f = h->solver->grid.fdtd;
    auto &g = f.grids[f.t + rel];
    return guarded([&] {
        cudaMemcpy(out, g.data.data(), sizeof(float) * g.data.size(), cudaMemcpyDeviceToHost);
        return last_cuda_status();
    });
}

int ref_cells_fresh_error(void *p)
{
    RefCells *h = (RefCells *)p;
    if (!h)
        return -1;
    auto e = h->solver->fresh_error.cpu();
    return e[0];
}

// ---- the reference GhostCellSolver as a whole (ghost_cell.h:72-152): set_mesh builds labels and
// the ghost system, each step is update(acc) (FDTD step, boundary condition, ghost solve, SOLID
// cells zeroed).  Handles share RefCells; threshold as set_condition_number_threshold.
void *ref_ghost_create(int res, float dl, float dt, const float *min_pos, float threshold)
{
    RefCells *h = (RefCells *)ref_cells_create(res, dl, dt, min_pos);
    if (h)
        h->solver->set_condition_number_threshold(threshold);
    return h;
}

int ref_ghost_set_mesh(void *p, const float *V, int nv, const int *F, int nt)
{
    RefCells *h = (RefCells *)p;
    if (!h || nv <= 0 || nt <= 0)
        return REF_ERR_ARG;
    int rc = h->cap.check(V, nv, F, nt, false);
    if (rc)
        return rc;
    h->nv = nv;
    h->nt = nt;
    return guarded([&] {
        CArr<float3> verts = to_float3(V, nv);
        CArr<int3> tris = to_int3(F, nt);
        h->solver->set_mesh(verts, tris);
        return last_cuda_status();
    });
}

int ref_ghost_update_mesh(void *p, const float *V)
{
    RefCells *h = (RefCells *)p;
    if (!h || h->nt == 0)
        return REF_ERR_STATE;
    return guarded([&] {
        CArr<float3> verts = to_float3(V, h->nv);
        h->solver->update_mesh(verts);
        return last_cuda_status();
    });
}

// nsteps steps with acc (nsteps x nt, host); the listener cells read after every step
int ref_ghost_run(void *p, const float *acc, int nsteps, const int *listen_xyz, int nlisten, float *out)
{
    RefCells *h = (RefCells *)p;
    if (!h || h->nt == 0 || nsteps < 0)
        return REF_ERR_ARG;
    return guarded([&] {
        auto &s = *h->solver;
        CArr<float> a(h->nt);
        for (int k = 0; k < nsteps; k++)
        {
            for (int i = 0; i < h->nt; i++)
                a[i] = acc[(size_t)k * h->nt + i];
            GArr<float> ga(a);
            s.update(ga);
            ga.clear();
            auto g = s.get_grid().cpu();
            const int n = s.res();
            for (int l = 0; l < nlisten; l++)
                out[(size_t)k * nlisten + l] =
                    g.data[((size_t)listen_xyz[3 * l] * n + listen_xyz[3 * l + 1]) * n + listen_xyz[3 * l + 2]];
        }
        return last_cuda_status();
    });
}

// ghost count, then per ghost: cell coordinates (3 ints), order (0 first, 1 second), 8 weights
int ref_ghost_count(void *p)
{
    RefCells *h = (RefCells *)p;
    return h ? h->solver->ghost_cell_num : -1;
}

int ref_ghost_read(void *p, int *coords, int *order, float *weights)
{
    RefCells *h = (RefCells *)p;
    if (!h)
        return REF_ERR_ARG;
    return guarded([&] {
        auto &s = *h->solver;
        const int g = s.ghost_cell_num;
        if (g <= 0)
            return 0;
        auto cells = s.ghost_cells.cpu();
        auto ord = s.ghost_order.cpu();
        for (int i = 0; i < g; i++)
        {
            coords[3 * i] = cells[i].x;
            coords[3 * i + 1] = cells[i].y;
            coords[3 * i + 2] = cells[i].z;
            order[i] = ord[i] == AccuracyOrder::SECOND_ORDER ? 1 : 0;
        }
        if (s.condition_number_threshold > 0)
        {
            auto w = s.p_weight.cpu();
            for (size_t i = 0; i < (size_t)g * GHOST_CELL_NEIGHBOR_NUM; i++)
                weights[i] = w.data[i];
        }
        else
            for (size_t i = 0; i < (size_t)g * GHOST_CELL_NEIGHBOR_NUM; i++)
                weights[i] = 0;
        return last_cuda_status();
    });
}

}  // extern "C"
