// cli.cpp -- the GTS command line (src/main.cu:43-180) over the C ABI.
//
//   gts data_path query_or_update_path op_type op_param result_path [options]
//
// op_type 0 = kNN (op_param = k), 1 = range (op_param = radius),
// 2 = stream update (op_param = radius of the query ops).  The result file
// has the reference's layout (main.cu:89-163).  Options set what the
// reference fixes at compile time (tree.cuh:31-35, update.cuh:16):
//   --order O --max-size S --max-h H --dis-code D --infi-dis I
//   --max-in-size C --form plain|fast
//   --ids PREFIX   also write saveK / saveR style id and distance files
//                  (file.cuh:154-199) to PREFIX.ids / PREFIX.dis
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>
#include "gts_b200.h"

static void die(const char *what)
{
    fprintf(stderr, "%s: %s\n", what, gts_last_error());
    exit(1);
}

int main(int argc, char **argv)
{
    if (argc < 6) {
        fprintf(stderr,
                "usage: %s data_path query_or_update_path op_type op_param result_path [--order O] "
                "[--max-size S] [--max-h H] [--dis-code D] [--infi-dis I] [--max-in-size C] "
                "[--form plain|fast] [--ids PREFIX]\n",
                argv[0]);
        return 2;
    }
    gts_params p;
    gts_params_default(&p);
    int form = GTS_FORM_PLAIN;
    const char *ids_prefix = nullptr;
    for (int i = 6; i + 1 < argc; i += 2) {
        std::string a = argv[i];
        int v = atoi(argv[i + 1]);
        if (a == "--order") p.tree_order = v;
        else if (a == "--max-size") p.max_size = v;
        else if (a == "--max-h") p.max_h = v;
        else if (a == "--dis-code") p.dis_code = v;
        else if (a == "--infi-dis") p.infi_dis = v;
        else if (a == "--max-in-size") p.max_in_size = v;
        else if (a == "--form") form = std::string(argv[i + 1]) == "fast" ? GTS_FORM_FAST : GTS_FORM_PLAIN;
        else if (a == "--ids") ids_prefix = argv[i + 1];
        else {
            fprintf(stderr, "unknown option %s\n", argv[i]);
            return 2;
        }
    }
    const int op = atoi(argv[3]);

    printf("Loading data file...\n");
    int dim, num, metric;
    float *rows = nullptr;
    char *strs = nullptr;
    int *lens = nullptr;
    if (gts_load(argv[1], &dim, &num, &metric, &rows, &strs, &lens) != GTS_OK) die("load");
    int *qids = nullptr, *flags = nullptr, *uids = nullptr, qnum = 0, nops = 0;
    int k = 0;
    float r = 0;
    if (op != 2) {
        printf("Loading query file...\n");
        if (gts_load_queries(argv[2], &qids, &qnum) != GTS_OK) die("loadQuery");
        k = atoi(argv[4]);
        r = (float)strtod(argv[4], nullptr);
    } else {
        printf("Loading update file...\n");
        if (gts_load_updates(argv[2], &flags, &uids, &nops) != GTS_OK) die("loadUpdate");
        r = (float)strtod(argv[4], nullptr);
    }

    printf("Index construction...\n");
    auto s = std::chrono::high_resolution_clock::now();
    gts_index *idx = nullptr;
    if (gts_index_build(dim, num, metric, rows, strs, lens, &p, &idx) != GTS_OK) die("indexConstru");
    auto e = std::chrono::high_resolution_clock::now();
    float time_index = std::chrono::duration<float>(e - s).count();
    gts_index_info info;
    gts_index_info_get(idx, &info);
    printf("Tree height: %d\n", info.tree_h);

    FILE *fcost = fopen(argv[5], "w");
    if (!fcost) {
        fprintf(stderr, "open file error: %s\n", argv[5]);
        return 1;
    }
    if (op == 0) {
        fprintf(fcost, "Knn search num: %d\nResult radius: \n", k);
        std::vector<float> kth(qnum);
        std::vector<int> ids;
        std::vector<float> dis;
        if (ids_prefix) {
            ids.resize((size_t)qnum * k);
            dis.resize((size_t)qnum * k);
        }
        printf("Searching...\n");
        s = std::chrono::high_resolution_clock::now();
        if (gts_knn(idx, qids, qnum, k, form, kth.data(), ids_prefix ? ids.data() : nullptr,
                    ids_prefix ? dis.data() : nullptr) != GTS_OK)
            die("searchIndexKnnV2");
        e = std::chrono::high_resolution_clock::now();
        float time_search = std::chrono::duration<float>(e - s).count();
        for (int i = 0; i < qnum; i++) fprintf(fcost, "%f ", kth[i]);
        printf("Time of index construction: %f\n", time_index);
        printf("Search time: %f\n", time_search / qnum);
        fprintf(fcost, "\nTime of index construction: %f\n", time_index);
        fprintf(fcost, "Search time: %f\n", time_search / qnum);
        if (ids_prefix) {   // saveK layout (file.cuh:154-176)
            std::string a = std::string(ids_prefix) + ".ids", b = std::string(ids_prefix) + ".dis";
            FILE *fr = fopen(a.c_str(), "w"), *fd = fopen(b.c_str(), "w");
            for (int i = 0; i < qnum; i++) {
                for (int j = 0; j < k; j++) {
                    fprintf(fr, "%d ", ids[(size_t)i * k + j]);
                    fprintf(fd, "%f ", dis[(size_t)i * k + j]);
                }
                fprintf(fr, "\n");
                fprintf(fd, "\n");
            }
            fclose(fr);
            fclose(fd);
        }
    } else if (op == 1) {
        fprintf(fcost, "Range search radius: %f\nResult num: \n", r);
        std::vector<int> counts(qnum);
        printf("Searching...\n");
        s = std::chrono::high_resolution_clock::now();
        if (gts_range_form(idx, qids, qnum, r, form, counts.data()) != GTS_OK) die("searchIndexRnnV2");
        e = std::chrono::high_resolution_clock::now();
        float time_search = std::chrono::duration<float>(e - s).count();
        for (int i = 0; i < qnum; i++) fprintf(fcost, "%d ", counts[i]);
        printf("\nTime of index construction: %f\n", time_index);
        printf("Search time: %f\n", time_search / qnum);
        fprintf(fcost, "\nTime of index construction: %f\n", time_index);
        fprintf(fcost, "Search time: %f\n", time_search / qnum);
        if (ids_prefix) {   // saveR layout (file.cuh:178-199)
            size_t total = 0;
            for (int c : counts) total += (size_t)c;
            std::vector<int> offs(qnum), rid(total + 1);
            std::vector<float> rdis(total + 1);
            if (gts_range_ids(idx, qids, qnum, r, counts.data(), offs.data(), rid.data(), rdis.data(), total) !=
                GTS_OK)
                die("range ids");
            std::string a = std::string(ids_prefix) + ".ids", b = std::string(ids_prefix) + ".dis";
            FILE *fr = fopen(a.c_str(), "a"), *fd = fopen(b.c_str(), "a");
            for (int i = 0; i < qnum; i++) {
                for (int j = offs[i]; j < offs[i] + counts[i]; j++) {
                    fprintf(fr, "%d ", rid[j]);
                    fprintf(fd, "%f ", rdis[j]);
                }
                fprintf(fr, "\n");
                fprintf(fd, "\n");
            }
            fclose(fr);
            fclose(fd);
        }
    } else {
        fprintf(fcost, "Range search radius (check for updates): %f\nResult num: \n", r);
        int nq_ops = 0;
        for (int i = 0; i < nops; i++) nq_ops += flags[i] == 2;
        std::vector<int> counts(nq_ops > 0 ? nq_ops : 1);
        int nq = 0;
        double ts = 0, tu = 0;
        printf("Updating...\n");
        if (gts_update_run(idx, flags, uids, nops, r, counts.data(), &nq, &ts, &tu) != GTS_OK)
            die("updateIndexRnn");
        for (int i = 0; i < nq; i++) fprintf(fcost, "%d ", counts[i]);
        int cnt_s = nq, cnt_u = nops - nq;
        float avg_s = cnt_s ? (float)(ts / cnt_s) : 0.f, avg_u = cnt_u ? (float)(tu / cnt_u) : 0.f;
        printf("Time of index construction: %f\n", time_index);
        printf("Total update time: %f\n", avg_s + avg_u);
        printf("Search time in update: %f\n", avg_s);
        printf("Update time in update: %f\n", avg_u);
        fprintf(fcost, "\nTime of index construction: %f\n", time_index);
        fprintf(fcost, "Total update time: %f\n", avg_s + avg_u);
        fprintf(fcost, "Search time in update : % f\n", avg_s);
        fprintf(fcost, "Update time in update: %f\n", avg_u);
    }
    fclose(fcost);
    gts_index_free(idx);
    gts_free_host(rows);
    gts_free_host(strs);
    gts_free_host(lens);
    gts_free_host(qids);
    gts_free_host(flags);
    gts_free_host(uids);
    return 0;
}
