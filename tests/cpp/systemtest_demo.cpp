// A GAT-style host program on the C++ layer (include/gat_b200.hpp): builds the three indexes over
// a seeded synthetic set, runs the SystemTest entry points and the batch forms, and prints every
// result as "name count v0 v1 ..." lines for the test that checks them against the oracle.
//
//   systemtest_demo <device> <n_trajectories> [trajectory file to write and read back]
//
// device < 0 runs host-only: the indexes are built, the queries return GAT_ERR_STATE.
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "gat_b200.hpp"

template <class T>
static void emit(const char* name, const std::vector<T>& v) {
    printf("%s %zu", name, v.size());
    for (const T& x : v) printf(" %lld", (long long)x);
    printf("\n");
}

int main(int argc, char** argv) {
    const int device = argc > 1 ? atoi(argv[1]) : 0;
    const int n = argc > 2 ? atoi(argv[2]) : 2000;
    const float box[4] = {121.0f, 30.7f, 122.0f, 31.7f};
    std::vector<int32_t> len(n);
    if (gat_gen_lengths(n, GAT_LEN_UNIFORM, 0, 0, 20, 200, 0, len.data()) != GAT_OK) return 2;
    int64_t total = 0;
    for (int v : len) total += v;
    std::vector<float> lon(total), lat(total);
    if (gat_gen_walks(n, len.data(), box, 1e-4, 0, lon.data(), lat.data()) != GAT_OK) return 2;
    // tradb[1..n], the reference's convention
    std::vector<gat::Trajectory> tradb(n + 1);
    int64_t o = 0;
    for (int t = 1; t <= n; t++) {
        tradb[t].tid = t;
        for (int i = 0; i < len[t - 1]; i++, o++) tradb[t].addSamplePoints(lon[o], lat[o], i);
    }
    if (argc > 3) {
        /* the reference's file format: write, read back, and read back the rewritten file */
        const gat::MBB box_mbb(box[0], box[1], box[2], box[3]);
        std::vector<gat::Trajectory> back, again;
        gat::MBB r1, r2;
        const std::string p2 = std::string(argv[3]) + ".2";
        int rc = gat::writeTrajectoryFile(argv[3], tradb.data(), n, box_mbb);
        rc = rc ? rc : gat::readTrajectoryFile(argv[3], back, &r1);
        rc = rc ? rc : gat::writeTrajectoryFile(p2.c_str(), back.data(), n, r1);
        rc = rc ? rc : gat::readTrajectoryFile(p2.c_str(), again, &r2);
        bool same = rc == GAT_OK && (int)back.size() == n + 1;
        for (int t = 1; same && t <= n; t++) {
            same = back[t].points.size() == tradb[t].points.size() && again[t].points.size() == back[t].points.size();
            for (size_t i = 0; same && i < back[t].points.size(); i++)
                same = back[t].points[i].lon == again[t].points[i].lon && back[t].points[i].lat == again[t].points[i].lat &&
                       back[t].points[i].time == (int)i;
        }
        printf("file_roundtrip %d\n", same ? 1 : 0);
    }
    try {
        gat::Context ctx(device);
        ctx.setTuning(GAT_TUNE_TOPK_GROWTH, 3);
        printf("tuning %d\n", ctx.tuning(GAT_TUNE_TOPK_GROWTH));
        ctx.setTuning(GAT_TUNE_TOPK_GROWTH, 0);
        const gat::MBB range(box[0], box[1], box[2], box[3]);
        gat::Grid g(ctx, range, 0.01f, 2, 512);
        gat::STIG stig(ctx);
        gat::FSG fsg(ctx, range, 0.01f);
        int rc = g.addDatasetToGrid(tradb.data(), n);
        rc = rc ? rc : stig.initial(256, 2, tradb.data(), n);
        rc = rc ? rc : fsg.addDatasetToGrid(tradb.data(), n);
        printf("build %d\n", rc);
        if (rc) return 3;
        /* the MortonGrid needs a device (GAT_ERR_STATE on a host-only context) */
        gat::MortonGrid mgrid(ctx, range, 0.01f, 2, 512);
        const int mrc = mgrid.addDatasetToGrid(tradb.data(), n);
        printf("mortonbuild %d\n", mrc);
        gat::SystemTest st(tradb.data(), &g, &stig, &fsg, mrc == GAT_OK ? &mgrid : nullptr);
        st.verbose = false;
        st.epsilon = 5e-4;
        const gat::MBB q(121.40f, 31.00f, 121.45f, 31.06f);
        rc = st.rangeQueryTest(q, 3);
        printf("rangeQueryTest %d\n", rc);
        if (rc == GAT_OK) emit("grid_off", st.lastRange.offsets), emit("grid_ids", st.lastRange.tids);
        rc = st.STIGrangeQueryTest(q, 2);
        printf("STIGrangeQueryTest %d\n", rc);
        if (rc == GAT_OK) emit("stig_off", st.lastRange.offsets), emit("stig_ids", st.lastRange.tids);
        rc = st.FSGrangeQueryTest(q, 2);
        printf("FSGrangeQueryTest %d\n", rc);
        if (rc == GAT_OK) emit("fsg_off", st.lastRange.offsets), emit("fsg_ids", st.lastRange.tids);
        rc = st.rangeQueryTestWithoutMorton(q, 2);
        printf("rangeQueryTestWithoutMorton %d\n", rc);
        if (rc == GAT_OK) emit("nonmorton_ids", st.lastRange.tids);
        rc = st.MortonGridRangeQueryTest(q, 2);
        printf("MortonGridRangeQueryTest %d\n", rc);
        if (rc == GAT_OK) emit("mortongrid_ids", st.lastRange.tids);
        // batch form with point results
        std::vector<float> b4(4 * 16);
        if (gat_gen_boxes(16, GAT_SIDE_LOGUNIFORM, 0.002, 0.05, box, 5, b4.data()) != GAT_OK) return 2;
        std::vector<gat::MBB> qs(16);
        for (int i = 0; i < 16; i++) qs[i] = gat::MBB(b4[4 * i], b4[4 * i + 1], b4[4 * i + 2], b4[4 * i + 3]);
        gat::RangeResult pts;
        rc = st.rangeQueryBatch(&g, qs.data(), 16, GAT_RESULT_POINTS, pts);
        printf("rangeQueryBatch %d\n", rc);
        if (rc == GAT_OK) emit("pts_off", pts.offsets), emit("pts_tid", pts.tids), emit("pts_pidx", pts.pidx);
        // README form: trajectory 47 as the query, 2 copies, k = 8
        rc = st.similarityQueryTest(47, 2, 8);
        printf("similarityQueryTest %d\n", rc);
        if (rc == GAT_OK) emit("topk_ids", st.lastTopk.ids), emit("topk_dist", st.lastTopk.dist);
    } catch (const gat::Error& e) {
        printf("error %d %s\n", e.status, e.what());
        return 4;
    }
    return 0;
}
