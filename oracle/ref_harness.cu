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
