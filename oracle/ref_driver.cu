// ref_driver.cu -- harness around the reference GTS build (test infrastructure).
//
// Compiled by oracle/Makefile against the UNMODIFIED reference headers
// (Source Code/GTS/include/*.cuh, taken from the reference checkout at build
// time; nothing of them is copied into this repository).  It calls the
// reference's own entry points -- indexConstru (tree.cuh:332),
// searchIndexKnnV2 (search_v2.cuh:975), searchIndexRnnV2 (search_v2.cuh:780),
// updateIndexRnn (update.cuh:449) -- and differs from the reference main
// (src/main.cu:43-180) only in what the reference left commented out:
//   * TREE_ORDER / MAX_SIZE / MAX_H / MAX_IN_SIZE come from the command line
//     (main.cu:54-58, 67-76 are commented out in the reference); the
//     reference declares them __managed__, so the host sets them directly;
//   * the list-table budget: the reference takes half of the free device
//     memory (search_v2.cuh:799, 995) and its int-typed sizes overflow above
//     ~16 GB, so the harness first parks device memory until half of what is
//     left equals --budget-gb (the commented input_size hook, main.cu:59-60);
//   * binary data files (".bin": int32 dim, num, metric, then rows) load
//     straight into managed memory; text files go through the reference's
//     own load() (file.cuh:28).
// Outputs: the reference's result file layout (main.cu:89-163), plus
// optional dumps of the built tree and per-query results, and a JSON line
// with timings on stdout.
//
// Usage:
//   gts_ref_driver DATA QUERY_OR_UPDATE OP PARAM RESULT
//       [--order O] [--max-size S] [--max-h H] [--max-in-size I]
//       [--budget-gb G] [--dump-tree FILE] [--dump-res FILE] [--search-only]

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <cuda_runtime_api.h>
#include <device_launch_parameters.h>
#include "tree.cuh"
#include "file.cuh"
#include "search.cuh"
#include "update.cuh"
#include "search_v2.cuh"
#include "config.cuh"

static bool ends_with(const std::string &s, const char *suf)
{
	size_t n = strlen(suf);
	return s.size() >= n && s.compare(s.size() - n, n, suf) == 0;
}

static void load_bin(const char *path, int *&info, float *&rows)
{
	FILE *f = fopen(path, "rb");
	if (!f) { fprintf(stderr, "cannot open %s\n", path); exit(2); }
	int hdr[3];
	if (fread(hdr, sizeof(int), 3, f) != 3) { fprintf(stderr, "bad header\n"); exit(2); }
	cudaMallocManaged((void **)&info, 3 * sizeof(int));
	info[0] = hdr[0]; info[1] = hdr[1]; info[2] = hdr[2];
	size_t n = (size_t)hdr[0] * hdr[1];
	cudaMallocManaged((void **)&rows, n * sizeof(float));
	if (fread(rows, sizeof(float), n, f) != n) { fprintf(stderr, "short data\n"); exit(2); }
	fclose(f);
}

static void *park_memory(double budget_gb)
{
	if (budget_gb <= 0) return nullptr;
	size_t avail = 0, total = 0;
	cudaMemGetInfo(&avail, &total);
	size_t want_free = (size_t)(2.0 * budget_gb * (1ull << 30));
	if (avail <= want_free) return nullptr;
	size_t park = avail - want_free;
	void *p = nullptr;
	if (cudaMalloc(&p, park) != cudaSuccess) { cudaGetLastError(); return nullptr; }
	return p;
}

int main(int argc, char **argv)
{
	if (argc < 6) {
		fprintf(stderr, "usage: %s DATA QUERY_OR_UPDATE OP PARAM RESULT [options]\n", argv[0]);
		return 2;
	}
	// keep the local-memory reservation of the edit-distance kernels
	// (int table[109][109] per thread) once made, so the parked memory below
	// does not starve later launches
	cudaSetDeviceFlags(cudaDeviceLmemResizeToMax);
	int op = atoi(argv[3]);
	double budget_gb = 6.0;
	int repeat = 1;
	const char *dump_tree = nullptr, *dump_res = nullptr;
	for (int i = 6; i + 1 < argc; i += 2) {
		std::string a = argv[i];
		if (a == "--order") TREE_ORDER = atoi(argv[i + 1]);
		else if (a == "--max-size") MAX_SIZE = atoi(argv[i + 1]);
		else if (a == "--max-h") MAX_H = atoi(argv[i + 1]);
		else if (a == "--max-in-size") MAX_IN_SIZE = atoi(argv[i + 1]);
		else if (a == "--budget-gb") budget_gb = atof(argv[i + 1]);
		else if (a == "--dump-tree") dump_tree = argv[i + 1];
		else if (a == "--dump-res") dump_res = argv[i + 1];
		else if (a == "--repeat") repeat = atoi(argv[i + 1]) > 0 ? atoi(argv[i + 1]) : 1;
		else { fprintf(stderr, "unknown option %s\n", argv[i]); return 2; }
	}

	int *data_info = nullptr;
	float *data_d = nullptr;
	char *data_s = nullptr;
	int *size_s = nullptr;
	std::string dpath = argv[1];
	if (ends_with(dpath, ".bin")) load_bin(argv[1], data_info, data_d);
	else load(argv[1], data_info, data_d, data_s, size_s);

	int *qid_list = nullptr;
	int qnum = 0;
	int k = 0;
	float r = 0;
	if (op != 2) {
		loadQuery(argv[2], qid_list, qnum);
		k = atoi(argv[4]);
		r = (float)std::stod(argv[4]);
	} else {
		loadUpdate(argv[2], update_list, update_num);
		r = (float)std::stod(argv[4]);
	}

	int *max_node_num = nullptr, *id_list = nullptr, *empty_list = nullptr;
	TN *node_list = nullptr;
	int tree_h = 0;
	cudaDeviceSynchronize();
	auto s = std::chrono::high_resolution_clock::now();
	indexConstru(data_d, data_s, size_s, data_info, id_list, node_list, max_node_num, tree_h, empty_list);
	cudaDeviceSynchronize();
	auto e = std::chrono::high_resolution_clock::now();
	double t_build = std::chrono::duration<double>(e - s).count();

	if (dump_tree) {
		int mnn = max_node_num[0];
		int n = data_info[1];
		int *h_id = (int *)malloc(sizeof(int) * n);
		TN *h_nodes = (TN *)malloc(sizeof(TN) * mnn);
		int *h_empty = (int *)malloc(sizeof(int) * mnn);
		cudaMemcpy(h_id, id_list, sizeof(int) * n, cudaMemcpyDeviceToHost);
		cudaMemcpy(h_nodes, node_list, sizeof(TN) * mnn, cudaMemcpyDeviceToHost);
		cudaMemcpy(h_empty, empty_list, sizeof(int) * mnn, cudaMemcpyDeviceToHost);
		FILE *f = fopen(dump_tree, "wb");
		int hdr[4] = {n, mnn, tree_h, start_idx};
		fwrite(hdr, sizeof(int), 4, f);
		fwrite(h_id, sizeof(int), n, f);
		for (int i = 0; i < mnn; i++) {
			int exists = h_empty[i] == 0;
			int rec[6];
			rec[0] = exists ? h_nodes[i].pid : 0;
			memcpy(&rec[1], &h_nodes[i].min_dis, 4);
			if (!exists) rec[1] = 0;
			rec[2] = exists ? h_nodes[i].size : 0;
			rec[3] = exists ? h_nodes[i].lid : 0;
			rec[4] = exists ? h_nodes[i].is_leaf : 0;
			rec[5] = exists;
			fwrite(rec, sizeof(int), 6, f);
		}
		fclose(f);
		free(h_id); free(h_nodes); free(h_empty);
	}

	void *parked = park_memory(budget_gb);
	FILE *fcost = fopen(argv[5], "w");
	double t_search = 0;
	std::string runs;
	if (op == 0) {
		fprintf(fcost, "Knn search num: %d\nResult radius: \n", k);
		for (int rep = 0; rep < repeat; rep++) {
			if (rep > 0) {
				// one search per process in the reference: its update_disk
				// global (search_v2.cuh:35) stays true after a call and res_dis
				// is allocated by every call
				update_disk = false;
				cudaFree(res_dis);
			}
			cudaDeviceSynchronize();
			s = std::chrono::high_resolution_clock::now();
			searchIndexKnnV2(data_d, node_list, id_list, max_node_num, qid_list, qnum, k, tree_h, data_info, empty_list, data_s, size_s);
			cudaDeviceSynchronize();
			e = std::chrono::high_resolution_clock::now();
			t_search = std::chrono::duration<double>(e - s).count();
			char buf[64];
			snprintf(buf, sizeof(buf), "%s%.6f", rep ? ", " : "", t_search);
			runs += buf;
		}
		for (int i = 0; i < qnum; i++) fprintf(fcost, "%f ", res_dis[i]);
		fprintf(fcost, "\nTime of index construction: %f\n", t_build);
		fprintf(fcost, "Search time: %f\n", t_search / qnum);
		if (dump_res) {
			FILE *f = fopen(dump_res, "wb");
			fwrite(res_dis, sizeof(float), qnum, f);
			fclose(f);
		}
	} else if (op == 1) {
		fprintf(fcost, "Range search radius: %f\nResult num: \n", r);
		for (int rep = 0; rep < repeat; rep++) {
			if (rep > 0) cudaFree(res);
			cudaDeviceSynchronize();
			s = std::chrono::high_resolution_clock::now();
			searchIndexRnnV2(data_d, node_list, id_list, max_node_num, qid_list, qnum, r, tree_h, data_info, empty_list, data_s, size_s);
			cudaDeviceSynchronize();
			e = std::chrono::high_resolution_clock::now();
			t_search = std::chrono::duration<double>(e - s).count();
			char buf[64];
			snprintf(buf, sizeof(buf), "%s%.6f", rep ? ", " : "", t_search);
			runs += buf;
		}
		for (int i = 0; i < qnum; i++) fprintf(fcost, "%d ", res[i]);
		fprintf(fcost, "\nTime of index construction: %f\n", t_build);
		fprintf(fcost, "Search time: %f\n", t_search / qnum);
		if (dump_res) {
			FILE *f = fopen(dump_res, "wb");
			fwrite(res, sizeof(int), qnum, f);
			fclose(f);
		}
	} else {
		fprintf(fcost, "Range search radius (check for updates): %f\nResult num: \n", r);
		int *qresult_count = nullptr, *qresult_count_prefix = nullptr, *result_id = nullptr;
		float *result_dis = nullptr;
		float t_us = 0, t_uu = 0;
		int c_us = 0, c_uu = 0;
		cudaDeviceSynchronize();
		s = std::chrono::high_resolution_clock::now();
		updateIndexRnn(data_d, node_list, id_list, max_node_num, qid_list, 1, r, tree_h, data_info, empty_list,
					   qresult_count, qresult_count_prefix, result_id, result_dis, data_s, size_s, fcost, t_us, t_uu,
					   c_us, c_uu);
		cudaDeviceSynchronize();
		e = std::chrono::high_resolution_clock::now();
		t_search = std::chrono::duration<double>(e - s).count();
		fprintf(fcost, "\nTime of index construction: %f\n", t_build);
		fprintf(fcost, "Total update time: %f\n", t_us / c_us + t_uu / c_uu);
		fprintf(fcost, "Search time in update : % f\n", t_us / c_us);
		fprintf(fcost, "Update time in update: %f\n", t_uu / c_uu);
		qnum = update_num;
	}
	fclose(fcost);
	if (parked) cudaFree(parked);
	cudaError_t err = cudaGetLastError();
	printf("{\"op\": %d, \"n\": %d, \"qnum\": %d, \"tree_h\": %d, \"build_s\": %.6f, \"search_s\": %.6f, "
		   "\"search_runs\": [%s], \"cuda\": \"%s\"}\n",
		   op, data_info[1], qnum, tree_h, t_build, t_search, runs.c_str(), cudaGetErrorString(err));
	return err == cudaSuccess ? 0 : 1;
}
