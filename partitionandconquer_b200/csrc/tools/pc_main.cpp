// pc_main -- the reference's CLI driver (src/test.cpp:301-390) and preprocess
// tool (src/preprocess.cpp) on the GPU library: same tasks, positional
// arguments, file layout (<graph_dir>/origin/csr_*.bin,
// <graph_dir>/partition/<method>/P<k>.bin) and output lines.
//
//   pc_main partition <graph_dir> <P> <out_dir>
//   pc_main generate_queries <num> <out_file>
//   pc_main bfs  <graph_dir> <is_partition> <method> <P> <threads>
//   pc_main cdlp <graph_dir> <is_partition> <method> <threads> <max_iteration>
//   pc_main kcore|mis|sssp <graph_dir> <is_partition> <method> <P> <threads>
//   pc_main tc   <graph_dir> <merge|galloping> <is_partition> <method> <P> <threads>
//   pc_main pr   <graph_dir> <is_partition> <method> <P> <threads> <damping> <iterations>
//   pc_main preprocess <graph_dir>/ <graph_file>
#include <algorithm>
#include <chrono>
#include <climits>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <numeric>
#include <memory>
#include <string>
#include <vector>

#include "../../../include/pc_graph.hpp"

using namespace std;
using pc::Graph;
using pc::Partitioned_Graph;

namespace {

// time_counter (src/Graph.cpp:5-25): accumulate and print with the same units.
struct Timer {
    chrono::high_resolution_clock::time_point t0;
    unsigned long long ns = 0;
    void start() { t0 = chrono::high_resolution_clock::now(); }
    void stop() { ns += chrono::duration_cast<chrono::nanoseconds>(chrono::high_resolution_clock::now() - t0).count(); }
    void print(const string& s) const {
        if (ns < 1000) printf("Time used for %s: %llu ns.\n", s.c_str(), ns);
        else if (ns < 1000000) printf("Time used for %s: %.3f us.\n", s.c_str(), (float)ns / 1000);
        else if (ns < 1000000000ull) printf("Time used for %s: %.3f ms.\n", s.c_str(), (float)ns / 1000000);
        else printf("Time used for %s: %.3f s.\n", s.c_str(), (float)ns / 1e9f);
    }
};

template <class T>
vector<T> read_vector(const string& f) {
    ifstream in(f, ios::binary);
    if (!in) {
        fprintf(stderr, "Error: cannot open binfile %s\n", f.c_str());
        exit(1);
    }
    in.seekg(0, ios::end);
    streamsize size = in.tellg();
    in.seekg(0, ios::beg);
    vector<T> v(size / sizeof(T));
    in.read(reinterpret_cast<char*>(v.data()), size);
    return v;
}

template <class T>
void save_vector(const vector<T>& v, const string& f) {
    ofstream out(f, ios::binary);
    out.write(reinterpret_cast<const char*>(v.data()), v.size() * sizeof(T));
}

string pfile(const string& dir, const string& method, int P) {
    return dir + "/partition/" + method + "/P" + to_string(P) + ".bin";
}

// The value the reference's serial k-core prints as "largest core"
// (Graph::solve_kcore, src/Graph.cpp:681-718): k - 1 at the first level k
// that finds no vertex left.  That is max core + 1 -- except when every
// vertex of the max core C has exactly max-core neighbours in C, so the whole
// of C goes in the first pass of its level and the next level never starts
// (then max core) -- and 0 when the peeling never finishes (a complete
// graph: the loop stops at k = n - 1 and every core reads 0, so a vertex of
// positive degree has core 0).  The core numbers themselves are exact.
int reference_largest_core_line(const Graph& g, const vector<int>& core) {
    const int n = g.get_vertex_num();
    if (n == 0) return 0;
    const pc::EID* vl = g.get_csr_vlist();
    const pc::VID* el = g.get_csr_elist();
    int mx = 0;
    for (int u = 0; u < n; ++u) {
        if (core[u] == 0 && vl[u + 1] > vl[u]) return 0;
        mx = max(mx, core[u]);
    }
    for (int u = 0; u < n; ++u) {
        if (core[u] != mx) continue;
        int inside = 0;
        for (pc::EID j = vl[u]; j < vl[u + 1]; ++j) inside += core[el[j]] == mx;
        if (inside != mx) return mx + 1;
    }
    return mx;
}

void head(const char* what, const vector<int>& v) {
    for (size_t i = 0; i < min<size_t>(10, v.size()); ++i) printf("  vertex: %zu, %s: %d\n", i, what, v[i]);
    printf("  ... \n");
}

int run(int argc, char** argv) {
    if (argc < 2) {
        fprintf(stderr, "usage: pc_main <task> ...\n");
        return 2;
    }
    const string task = argv[1];
    auto need = [&](int k) {
        if (argc < k) {
            fprintf(stderr, "task %s needs %d arguments\n", task.c_str(), k - 2);
            exit(2);
        }
    };
    Timer t;
    if (task == "partition") {
        need(5);
        const string dir = argv[2], out = argv[4];
        const size_t P = stoul(argv[3]);
        Graph g(dir + "/origin", false);
        vector<int> v2p;
        t.start();
        g.greedy_partition(P, v2p);
        t.stop();
        t.print("greedy partition");
        Partitioned_Graph G(g, v2p, (int)P);
        G.evaluate_partition();
        save_vector(v2p, out + "/P" + to_string(P) + ".bin");
    } else if (task == "generate_queries") {
        need(4);
        const size_t q = stoul(argv[2]);
        vector<int> qs;
        for (size_t i = 0; i < q; ++i) {
            qs.push_back(rand());
            qs.push_back(rand());
        }
        save_vector(qs, argv[3]);
    } else if (task == "preprocess") {
        // src/preprocess.cpp:39-45: text -> <dir>/origin CSR files + weights
        need(4);
        const string dir = argv[2], file = argv[3];
        // the adjacency build runs on the GPU when there is one (same arrays)
        std::unique_ptr<Graph> gp = pc_device_count() > 0 ? std::make_unique<Graph>(dir + file, Graph::OnDevice{})
                                                           : std::make_unique<Graph>(dir + file);
        Graph& g = *gp;
        printf("Number of nodes: %d, number of edges: %llu.\n", g.get_vertex_num(), g.get_edge_num());
        g.save_as_csr_binfile(dir + "/origin/csr_vlist.bin", dir + "/origin/csr_elist.bin");
        g.add_reference_weights();
        g.save_weight_binfile(dir + "/origin/csr_weight.bin");
    } else if (task == "bfs" || task == "kcore" || task == "mis" || task == "sssp") {
        need(7);
        const string dir = argv[2], method = argv[4];
        const bool part = stod(argv[3]) != 0;
        const int P = (int)stod(argv[5]), threads = (int)stod(argv[6]);
        Graph g(dir + "/origin", task == "sssp");
        const int n = g.get_vertex_num();
        vector<int> v2p;
        if (part) v2p = read_vector<int>(pfile(dir, method, P));
        Partitioned_Graph G(g, v2p, threads);
        G.solve_triangle_counting_merge();  // plan / warm the device outside the timer
        vector<int> res;
        if (task == "bfs") {
            t.start();
            G.solve_bfs(0, res);
            t.stop();
            t.print(part ? "partitioned BFS" : "serial BFS");
            printf("Vertex Rank: \n");
            head("rank", res);
        } else if (task == "kcore") {
            t.start();
            G.solve_kcore(res);
            t.stop();
            printf("largest core: %d.\n", reference_largest_core_line(g, res));
            t.print(part ? "partitioned Core Decomposition" : "parallel Core Decomposition");
        } else if (task == "mis") {
            t.start();
            G.solve_mis(res);
            t.stop();
            t.print(part ? "partitioned MIS" : "parallel MIS");
            printf("Size of independent set: %d\n", accumulate(res.begin(), res.end(), 0));
        } else {
            t.start();
            G.solve_sssp(0, res);
            t.stop();
            t.print(part ? "partitioned SSSP" : "parallel SSSP");
            int mx = 0;
            for (int u = 0; u < n; ++u)
                if (res[u] != INT_MAX / 2 && res[u] > mx) mx = res[u];
            printf("Max distance: %d\n", mx);
            printf("Vertex distances: \n");
            head("distance", res);
        }
    } else if (task == "cdlp") {
        need(7);
        const string dir = argv[2], method = argv[4];
        const bool part = stod(argv[3]) != 0;
        const int threads = stoi(argv[5]), iters = stoi(argv[6]);
        Graph g(dir + "/origin", false);
        const int n = g.get_vertex_num();
        vector<int> labels(n);
        iota(labels.begin(), labels.end(), 0);
        vector<int> v2p;
        // src/test.cpp:123 names the partition file after num_threads
        if (part) v2p = read_vector<int>(pfile(dir, method, threads));
        Partitioned_Graph G(g, v2p, threads);
        t.start();
        G.solve_cdlp(labels, iters);
        t.stop();
        t.print(part ? "partitioned CDLP" : "parallel CDLP");
        printf("Vertex labels: \n");
        head("label", labels);
    } else if (task == "tc") {
        need(8);
        const string dir = argv[2], how = argv[3], method = argv[5];
        const bool part = stod(argv[4]) != 0;
        const int P = (int)stod(argv[6]), threads = (int)stod(argv[7]);
        Graph g(dir + "/origin", false);
        vector<int> v2p;
        if (part) v2p = read_vector<int>(pfile(dir, method, P));
        Partitioned_Graph G(g, v2p, threads);
        size_t res = 0;
        t.start();
        if (how == "merge") res = G.solve_triangle_counting_merge();
        else if (how == "galloping") res = G.solve_triangle_counting_galloping();
        t.stop();
        t.print((part ? "partitioned " : "paralle ") + how);
        printf("#Triangles: %zu.\n", res);
    } else if (task == "pr") {
        need(9);
        const string dir = argv[2], method = argv[4];
        const bool part = stod(argv[3]) != 0;
        const int P = stoi(argv[5]), threads = stoi(argv[6]), iters = stoi(argv[8]);
        const float damping = stof(argv[7]);
        Graph g(dir + "/origin", false);
        const int n = g.get_vertex_num();
        vector<float> pr(n, 1.0f);
        printf("Task information: #Threads = %d, Damping factor = %.3f, #Iterations = %d\n", threads, damping, iters);
        if (part) {
            Partitioned_Graph G(g, read_vector<int>(pfile(dir, method, P)), threads);
            G.reorder();
            t.start();
            G.page_rank(pr, damping, iters);
            t.stop();
            t.print("partitioned PageRank");
        } else {
            t.start();
            g.page_rank(pr, damping, iters, threads);
            t.stop();
            t.print("parallel PageRank");
        }
        if (n) {
            printf("Max PageRank: %f, Min PageRank: %f\n", *max_element(pr.begin(), pr.end()),
                   *min_element(pr.begin(), pr.end()));
            printf("PageRank values (head 10): \n");
            for (int i = 0; i < min(10, n); ++i) printf("  vertex: %d, pr_vals: %f .\n", i, pr[i]);
        }
    } else {
        fprintf(stderr, "unknown task %s\n", task.c_str());
        return 2;
    }
    return 0;
}

}  // namespace

int main(int argc, char** argv) {
    try {
        return run(argc, argv);
    } catch (const pc::Error& e) {
        fprintf(stderr, "pc error %d: %s\n", (int)e.status, e.what());
        return 1;
    }
}
