// tc_cli.cpp -- the `tc` command line tool on top of libwetric.
//
// Same flags and same output table as the reference's main (tc.cu:816-918):
//   -m <file> | -e <file>   Matrix Market / edge list input
//   -s <num>                spread (required, > 0)
//   -a <num>                bitmap length (multiple of 32, default 0)
//   -l <num>                loop count (default 1; one extra warm-up run
//                           is not printed)
//   -z                      zero-indexed input
//   -p <0|1|2>              preprocessing style (accepted; all run on GPU)
//   -j <file>               also append one JSON line per printed run to
//                           <file> (wedges, wedges/s, triangles/s, times)
// The pipeline is read_graph -> preprocess -> loop of tc_GPU, with each
// call replaced by its libwetric mirror. "prepro (s)" times the preprocess
// step only, as in the reference (tc.cu:886-888); "GPU copy" is the
// host->device copy of the CSR, "GPU exec" all device work of the count
// (wedge prefix, bitmap and count kernels), "CPU+GPU" the wall time of the
// whole count call.
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <sys/time.h>

#include "../../include/wetric.h"

static double wall_seconds() {
  struct timeval tv;
  gettimeofday(&tv, nullptr);
  return (double)tv.tv_sec + (double)tv.tv_usec / 1e6;
}

static void usage() {
  printf("Wedge-parallel triangle counting (B200)\n\n");
  printf("Usage:\n\n");
  printf("One input is required:\n");
  printf(" -m <filename>   input graph in Matrix Market format\n");
  printf(" -e <filename>   input graph as a text edge list\n");
  printf("Required:\n");
  printf(" -s <num>        spread: wedges per thread\n");
  printf(" -a <num>        bitmap length, a multiple of 32\n");
  printf(" -c <filename>   input graph as a binary CSR cache (written by -w)\n");
  printf("Optional:\n");
  printf(" -w <filename>   write the preprocessed graph as a binary CSR cache\n");
  printf(" -l <num>        loop count\n");
  printf(" -z              input graph is zero-indexed\n");
  printf(" -p <0|1|2>      preprocessing style (all styles run on the GPU)\n");
  printf(" -j <filename>   append one JSON line per run (wedges/s, triangles/s, times)\n");
  printf("\nExample:\n");
  printf("./tc -m graph.mtx -s 5 -a 8192 -l 10\n");
  exit(EXIT_FAILURE);
}

static void fail(const char *what) {
  fprintf(stderr, "ERROR: %s: %s (%s)\n", what,
          wetric_strerror(wetric_last_error()), wetric_last_error_message());
  exit(EXIT_FAILURE);
}

int main(int argc, char **argv) {
  char *filename = nullptr;
  char *cache_out = nullptr;
  char *json_out = nullptr;
  int mm = 0, zero_indexed = 0, from_cache = 0;
  unsigned loops = 1;
  int style = WETRIC_PREPROCESS_GPU_CONSTRAINED;
  unsigned spread = 0, alen = 0;

  while (argc > 1 && argv[1][0] == '-') {
    switch (argv[1][1]) {
      case 'm':
        mm = 1;
        /* fall through: -m is -e with the Matrix Market flag */
      case 'e':
        if (argc < 3) usage();
        filename = argv[2];
        argv += 2;
        argc -= 2;
        break;
      case 'c':
        if (argc < 3) usage();
        filename = argv[2];
        from_cache = 1;
        argv += 2;
        argc -= 2;
        break;
      case 'w':
        if (argc < 3) usage();
        cache_out = argv[2];
        argv += 2;
        argc -= 2;
        break;
      case 'j':
        if (argc < 3) usage();
        json_out = argv[2];
        argv += 2;
        argc -= 2;
        break;
      case 'z':
        zero_indexed = 1;
        argv++;
        argc--;
        break;
      case 'a':
        if (argc < 3) usage();
        alen = (unsigned)atoi(argv[2]);
        if (alen % 32 != 0) usage();
        argv += 2;
        argc -= 2;
        break;
      case 's':
        if (argc < 3) usage();
        if (atoi(argv[2]) <= 0) usage();
        spread = (unsigned)atoi(argv[2]);
        argv += 2;
        argc -= 2;
        break;
      case 'l':
        if (argc < 3) usage();
        loops = (unsigned)atoi(argv[2]);
        argv += 2;
        argc -= 2;
        break;
      case 'p':
        if (argc < 3) usage();
        if (atoi(argv[2]) < 0 || atoi(argv[2]) > 2) usage();
        style = atoi(argv[2]);
        argv += 2;
        argc -= 2;
        break;
      default:
        usage();
    }
  }
  if (filename == nullptr || spread == 0) usage();

  wetric_big_graph *original = nullptr;
  bool oriented = false;
  if (from_cache) {
    // a cached CSR: already preprocessed when it was written oriented
    wetric_csr c;
    const int st = wetric_load_csr(filename, &c);
    if (st != WETRIC_OK) {
      fprintf(stderr, "ERROR: load_csr: %s (%s)\n", wetric_strerror(st), filename);
      exit(EXIT_FAILURE);
    }
    original = (wetric_big_graph *)malloc(sizeof(wetric_big_graph));
    if (!original) exit(EXIT_FAILURE);
    original->numVertices = (uint32_t)c.n;
    original->numEdges = c.m;
    original->rowPtr = (uint64_t *)c.row_ptr;
    original->colInd = (uint32_t *)c.col_ind;
    oriented = (c.flags & WETRIC_CSR_ORIENTED) != 0;
  } else {
    original = wetric_read_big_graph(filename, mm, zero_indexed, style);
    if (!original) fail("read_graph");
  }
  double t_pre = wall_seconds();
  wetric_big_graph *graph = original;
  if (!oriented) {
    graph = wetric_preprocess_big(original, style);
    if (!graph) fail("preprocess");
    wetric_free_big_graph(original);
  }
  t_pre = wall_seconds() - t_pre;
  if (cache_out) {
    wetric_csr c = {graph->numVertices, graph->numEdges, graph->rowPtr,
                    graph->colInd, WETRIC_CSR_ORIENTED};
    const int st = wetric_save_csr(cache_out, &c);
    if (st != WETRIC_OK) {
      fprintf(stderr, "ERROR: save_csr: %s (%s)\n", wetric_strerror(st), cache_out);
      exit(EXIT_FAILURE);
    }
  }

  FILE *jf = nullptr;
  uint64_t wedges = 0;
  if (json_out) {
    jf = fopen(json_out, "a");
    if (!jf) {
      fprintf(stderr, "ERROR: cannot open %s\n", json_out);
      exit(EXIT_FAILURE);
    }
    for (uint32_t v = 0; v < graph->numVertices; ++v) {
      const uint64_t d = graph->rowPtr[v + 1] - graph->rowPtr[v];
      wedges += d * (d ? d - 1 : 0) / 2;
    }
  }
  printf("%-60s %16s %16s %16s %16s %16s %16s %16s %16s %16s %16s\n", "graph",
         "n", "m", "s", "a", "triangles", "prepro (s)", "GPU copy (s)",
         "GPU exec (s)", "GPU total (s)", "CPU+GPU (s)");
  for (unsigned i = 0; i < loops + 1; ++i) {
    double t_cpu = wall_seconds();
    wetric_gpu_time t = {0.0, 0.0};
    const uint64_t tri = wetric_tc_gpu_big(graph, spread, alen, &t);
    t_cpu = wall_seconds() - t_cpu;
    if (tri == UINT64_MAX) fail("tc_GPU");
    t.copy /= 1000.0;
    t.exec /= 1000.0;
    if (i > 0) {
      printf("%-60s %16u %16llu %16u %16u %16llu %16.6f %16.6f %16.6f %16.6f "
             "%16.6f\n",
             filename, graph->numVertices, (unsigned long long)graph->numEdges,
             spread, alen, (unsigned long long)tri, t_pre, t.copy, t.exec,
             t.copy + t.exec, t_cpu);
      if (jf) {
        fprintf(jf,
                "{\"graph\": \"%s\", \"n\": %u, \"m\": %llu, \"s\": %u, \"a\": %u, "
                "\"triangles\": %llu, \"wedges\": %llu, \"prepro_s\": %.6f, "
                "\"copy_s\": %.6f, \"exec_s\": %.6f, \"cpu_gpu_s\": %.6f, "
                "\"wedges_per_s\": %.6e, \"triangles_per_s\": %.6e}\n",
                filename, graph->numVertices, (unsigned long long)graph->numEdges, spread,
                alen, (unsigned long long)tri, (unsigned long long)wedges, t_pre, t.copy,
                t.exec, t_cpu, t.exec > 0 ? (double)wedges / t.exec : 0.0,
                t.exec > 0 ? (double)tri / t.exec : 0.0);
      }
    }
  }
  if (jf) fclose(jf);
  wetric_free_big_graph(graph);
  return EXIT_SUCCESS;
}
