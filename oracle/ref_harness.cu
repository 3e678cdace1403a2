// ref_harness.cu -- drives the reference's own functions on a given input to
// produce golden vectors (test infrastructure; links the reference objects
// compiled from the reference tree, never part of the product).
//
//   ref_harness sweeps <file.mtx> <n> <out.bin>
//       readInputData + copyStructures + initM, then n calls of
//       optimiseModularity(1e30f): each call runs exactly one sweep (the loop
//       condition totalGain >= minGain holds once, modularity_optimisation.cu:341-343)
//       and copies vertexCommunity to the host.  out: int32 V, int32 n, then
//       n blocks of V int32 (communities after each sweep).
//   ref_harness sweeps1 <file.mtx> <n> <out.bin>
//       the same n sweeps, orchestrated here like optimiseModularity
//       (modularity_optimisation.cu:306-349: bucket sub-rounds, commit,
//       Sigma_tot rebuild), but launching the reference's own computeMoveShared
//       / computeMoveGlobal kernels with ONE thread per vertex (blockDim.x = 1).
//       The stock launch shape has a write race at
//       modularity_optimisation.cu:192-196 (every lane but 0 stores the old
//       community into the slot lane 0 writes); with one lane per vertex the
//       race cannot occur and the kernels compute the rule as written.
//   ref_harness aggregate <file.mtx> <comm.bin> <out.bin>
//       sets vertexCommunity and originalToCommunity to the given vector and
//       calls aggregateCommunities once.  out: int32 V', int32 E', int32 V0,
//       rowptr[V'+1], col[E'], float w[E'], int32 orig2comm[V0],
//       float communityWeight[V'].
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "community_aggregation.cuh"
#include "modularity_optimisation.cuh"
#include "utils.cuh"

// Host stubs of the reference's kernels (defined in modularity_optimisation.o);
// launched through cudaLaunchKernel with the stub address.
void computeEdgesSum(device_structures deviceStructures);
void computeCommunityWeight(device_structures deviceStructures);
void computeMoveShared(int V, int *vertices, int prime, device_structures deviceStructures);
void computeMoveGlobal(int V, int *vertices, int prime, device_structures deviceStructures,
                       int *hashCommunity, float *hashWeight);
void updateVertexCommunity(int V, int *vertices, device_structures deviceStructures);

static const int kBounds[8] = {0, 4, 8, 16, 32, 84, 319, INT_MAX};
static const int kPrimes[6] = {7, 13, 29, 53, 127, 479};

static int next_prime(int n) {
    for (;;) {
        ++n;
        bool p = n > 1;
        for (int i = 2; (long long)i * i <= n; ++i)
            if (n % i == 0) { p = false; break; }
        if (p) return n;
    }
}

static void sweep_one_lane(host_structures &hs, device_structures &ds, int *d_list) {
    const int V = hs.V;
    std::vector<int> rp(V + 1);
    HANDLE_ERROR(cudaMemcpy(rp.data(), ds.edgesIndex, sizeof(int) * (V + 1), cudaMemcpyDeviceToHost));
    for (int b = 0; b < 7; ++b) {
        std::vector<int> list;
        int maxdeg = 0;
        for (int v = 0; v < V; ++v) {
            int d = rp[v + 1] - rp[v];
            if (d > kBounds[b] && d <= kBounds[b + 1]) { list.push_back(v); maxdeg = d > maxdeg ? d : maxdeg; }
        }
        int n = (int)list.size();
        if (n == 0) continue;
        HANDLE_ERROR(cudaMemcpy(d_list, list.data(), sizeof(int) * n, cudaMemcpyHostToDevice));
        if (b < 6) {
            int prime = kPrimes[b];
            int y = 32;
            while (y > 1 && (size_t)y * prime * 8 + 4 * y > 48 * 1024) y /= 2;
            size_t smem = (size_t)y * prime * 8 + 4 * y;
            dim3 grid((n + y - 1) / y), block(1, y);
            void *args[] = {&n, &d_list, &prime, &ds};
            HANDLE_ERROR(cudaLaunchKernel((const void *)computeMoveShared, grid, block, args, smem, 0));
        } else {
            int prime = next_prime((int)(maxdeg * 1.5));
            int *hc = nullptr;
            float *hw = nullptr;
            HANDLE_ERROR(cudaMalloc((void **)&hc, sizeof(int) * (size_t)prime * n));
            HANDLE_ERROR(cudaMalloc((void **)&hw, sizeof(float) * (size_t)prime * n));
            dim3 grid(n), block(1, 1);
            size_t smem = THREADS_PER_BLOCK * (sizeof(int) + sizeof(float)) + sizeof(float);
            void *args[] = {&n, &d_list, &prime, &ds, &hc, &hw};
            HANDLE_ERROR(cudaLaunchKernel((const void *)computeMoveGlobal, grid, block, args, smem, 0));
            HANDLE_ERROR(cudaDeviceSynchronize());
            HANDLE_ERROR(cudaFree(hc));
            HANDLE_ERROR(cudaFree(hw));
        }
        {
            dim3 grid((n + THREADS_PER_BLOCK - 1) / THREADS_PER_BLOCK), block(THREADS_PER_BLOCK);
            void *args[] = {&n, &d_list, &ds};
            HANDLE_ERROR(cudaLaunchKernel((const void *)updateVertexCommunity, grid, block, args, 0, 0));
        }
        HANDLE_ERROR(cudaMemset(ds.communityWeight, 0, sizeof(float) * V));
        {
            dim3 grid((V + THREADS_PER_BLOCK - 1) / THREADS_PER_BLOCK), block(THREADS_PER_BLOCK);
            void *args[] = {&ds};
            HANDLE_ERROR(cudaLaunchKernel((const void *)computeCommunityWeight, grid, block, args, 0, 0));
        }
        HANDLE_ERROR(cudaDeviceSynchronize());
    }
}

static void write_all(FILE *f, const void *p, size_t n) {
    if (n && fwrite(p, 1, n, f) != n) {
        fprintf(stderr, "write failed\n");
        exit(2);
    }
}

int main(int argc, char **argv) {
    if (argc != 5) {
        fprintf(stderr, "usage: ref_harness sweeps|aggregate <mtx> <n|comm.bin> <out>\n");
        return 1;
    }
    std::string mode = argv[1];
    host_structures hs = readInputData(argv[2]);
    device_structures ds;
    aggregation_phase_structures as;
    copyStructures(hs, ds, as);
    initM(hs);
    FILE *out = fopen(argv[4], "wb");
    if (!out) return 2;
    if (mode == "sweeps") {
        int n = atoi(argv[3]);
        int V = hs.V;
        write_all(out, &V, 4);
        write_all(out, &n, 4);
        for (int s = 0; s < n; ++s) {
            optimiseModularity(1e30f, ds, hs);
            write_all(out, hs.vertexCommunity, sizeof(int) * (size_t)V);
        }
    } else if (mode == "sweeps1") {
        int n = atoi(argv[3]);
        int V = hs.V;
        write_all(out, &V, 4);
        write_all(out, &n, 4);
        int *d_list = nullptr;
        HANDLE_ERROR(cudaMalloc((void **)&d_list, sizeof(int) * (V > 0 ? V : 1)));
        {
            // k_i of the level (computeEdgesSum, modularity_optimisation.cu:286)
            dim3 grid((V * WARP_SIZE + THREADS_PER_BLOCK - 1) / THREADS_PER_BLOCK);
            dim3 block(WARP_SIZE, THREADS_PER_BLOCK / WARP_SIZE);
            void *args[] = {&ds};
            HANDLE_ERROR(cudaLaunchKernel((const void *)computeEdgesSum, grid, block, args, 0, 0));
            HANDLE_ERROR(cudaDeviceSynchronize());
        }
        std::vector<int> comm(V);
        for (int s = 0; s < n; ++s) {
            sweep_one_lane(hs, ds, d_list);
            HANDLE_ERROR(cudaMemcpy(comm.data(), ds.vertexCommunity, sizeof(int) * V, cudaMemcpyDeviceToHost));
            write_all(out, comm.data(), sizeof(int) * (size_t)V);
        }
        HANDLE_ERROR(cudaFree(d_list));
    } else if (mode == "aggregate") {
        int V = hs.V;
        std::vector<int> comm(V);
        FILE *cf = fopen(argv[3], "rb");
        if (!cf || fread(comm.data(), 4, (size_t)V, cf) != (size_t)V) return 3;
        fclose(cf);
        HANDLE_ERROR(cudaMemcpy(ds.vertexCommunity, comm.data(), sizeof(int) * V, cudaMemcpyHostToDevice));
        HANDLE_ERROR(cudaMemcpy(ds.originalToCommunity, comm.data(), sizeof(int) * V, cudaMemcpyHostToDevice));
        aggregateCommunities(ds, hs, as);
        HANDLE_ERROR(cudaDeviceSynchronize());
        int V2 = hs.V, E2 = hs.E, V0 = hs.originalV;
        std::vector<int> rp(V2 + 1), cl(E2 > 0 ? E2 : 1), o2c(V0);
        std::vector<float> wt(E2 > 0 ? E2 : 1), cw(V2 > 0 ? V2 : 1);
        HANDLE_ERROR(cudaMemcpy(rp.data(), ds.edgesIndex, sizeof(int) * (V2 + 1), cudaMemcpyDeviceToHost));
        HANDLE_ERROR(cudaMemcpy(cl.data(), ds.edges, sizeof(int) * E2, cudaMemcpyDeviceToHost));
        HANDLE_ERROR(cudaMemcpy(wt.data(), ds.weights, sizeof(float) * E2, cudaMemcpyDeviceToHost));
        HANDLE_ERROR(cudaMemcpy(o2c.data(), ds.originalToCommunity, sizeof(int) * V0, cudaMemcpyDeviceToHost));
        HANDLE_ERROR(cudaMemcpy(cw.data(), ds.communityWeight, sizeof(float) * V2, cudaMemcpyDeviceToHost));
        write_all(out, &V2, 4);
        write_all(out, &E2, 4);
        write_all(out, &V0, 4);
        write_all(out, rp.data(), sizeof(int) * (V2 + 1));
        write_all(out, cl.data(), sizeof(int) * E2);
        write_all(out, wt.data(), sizeof(float) * E2);
        write_all(out, o2c.data(), sizeof(int) * V0);
        write_all(out, cw.data(), sizeof(float) * V2);
    } else {
        return 1;
    }
    fclose(out);
    return 0;
}
