// `ngap` command line: a drop-in for the reference CLI
// (code/src/ngap/main.cu:16-137, options code/src/ngap/ngap_option.h:6-69 and
// code/include/commons/common_func.h:19-130). Same flags, same defaults, same
// stdout lines parsed by the reference's experiment scripts
// (code/scripts/launch_exps.py:443-458): "Results number", "Unique results
// number", "Validation PASS!/FAILED!", "ngap elapsed time: <s> seconds,
// throughput = <MB/s> MB/s", "FINISHED!". Matching runs on the GPU through the
// C ABI; --validation runs the library's CPU checker as the reference does.
#include <algorithm>
#include <cctype>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <functional>
#include <iostream>
#include <map>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/ngap_b200.h"

namespace {

struct Options {
  // common_gpunfa_options (common_func.h:50-58)
  int block_size = 256;
  std::string algorithm = "graph";
  std::string report_filename = "report.txt";
  int max_nfa_size = -1;
  int duplicate_input_stream = 1;
  int input_start_pos = 0;
  int input_len = -1;
  unsigned long long output_capacity = 54619400ull;
  bool report_off = false;
  bool show_help = false;
  int split_chunk_size = -1;
  std::string input_filename, nfa_filename, app_name, select_cc_by_state;
  int only_exec_cc = -1;
  int padding = 256;
  long long quick_validation = -1;
  int unique_frequency = 0;
  bool use_uvm = false, quit_degree = true, remove_degree = false;
  // ngap_option (ngap_option.h:52-68)
  unsigned data_buffer_fetch_size = 128;
  int add_aas_start = 0, add_aas_interval = 1;
  bool unique = false, validation = true;
  int active_threshold = 20;
  bool use_soa = false;
  int precompute_cutoff = -1, precompute_depth = 0;
  bool motivate_worklist_length = false;
  int num_state_per_group = 256;
  int group_num = 10;
  bool compress_prec_table = true, tuning = false, pc_use_uvm = false, adaptive_aas = false,
       try_adaptive_aas = false;
  // additions of this engine
  std::string dump_reports;  // binary dump of the sorted unique reports (u64 each)
  int window = 0, chunk = 0, tile_states = 0, tile_mode = 0;
};

bool parse_bool(const std::string& v, bool& out) {
  std::string s;
  for (char c : v) s.push_back((char)tolower((unsigned char)c));
  if (s == "true" || s == "1" || s == "yes" || s == "y" || s == "on") {
    out = true;
    return true;
  }
  if (s == "false" || s == "0" || s == "no" || s == "n" || s == "off") {
    out = false;
    return true;
  }
  return false;
}

template <class T>
bool parse_num(const std::string& v, T& out) {
  std::istringstream is(v);
  T x;
  if (!(is >> x)) return false;
  out = x;
  return true;
}

bool parse_args(int argc, char** argv, Options& o, std::string& err) {
  std::map<std::string, std::function<bool(const std::string&)>> h;
  auto b = [&](bool& f) { return [&f](const std::string& v) { return parse_bool(v, f); }; };
  auto i = [&](int& f) { return [&f](const std::string& v) { return parse_num(v, f); }; };
  auto s = [&](std::string& f) { return [&f](const std::string& v) { f = v; return true; }; };
  h["--algorithm"] = h["-g"] = s(o.algorithm);
  h["--block-size"] = i(o.block_size);
  h["--max-nfa-size"] = i(o.max_nfa_size);
  h["--report-off"] = b(o.report_off);
  h["--report-filename"] = s(o.report_filename);
  h["--result-capacity"] = [&](const std::string& v) { return parse_num(v, o.output_capacity); };
  h["--input-start-pos"] = i(o.input_start_pos);
  h["--input-len"] = i(o.input_len);
  h["--input"] = h["-i"] = s(o.input_filename);
  h["--automata"] = h["-a"] = s(o.nfa_filename);
  h["--split-entire-inputstream-to-chunk-size"] = i(o.split_chunk_size);
  h["--only-exec-cc-with-state-id"] = s(o.select_cc_by_state);
  h["--only-exec-ccid"] = i(o.only_exec_cc);
  h["--duplicate-input-stream"] = i(o.duplicate_input_stream);
  h["--quick-validation"] = [&](const std::string& v) { return parse_num(v, o.quick_validation); };
  h["--unique-frequency"] = i(o.unique_frequency);
  h["--padding"] = i(o.padding);
  h["--app-name"] = s(o.app_name);
  h["--use-uvm"] = b(o.use_uvm);
  h["--quit-degree"] = b(o.quit_degree);
  h["--remove-degree"] = b(o.remove_degree);
  h["--add-aan-start"] = i(o.add_aas_start);
  h["--add-aas-interval"] = i(o.add_aas_interval);
  h["--unique"] = b(o.unique);
  h["--active-threshold"] = i(o.active_threshold);
  h["--validation"] = b(o.validation);
  h["--use-soa"] = b(o.use_soa);
  h["--precompute-cutoff"] = i(o.precompute_cutoff);
  h["--precompute-depth"] = i(o.precompute_depth);
  h["--data-buffer-fetch-size"] = [&](const std::string& v) {
    return parse_num(v, o.data_buffer_fetch_size);
  };
  h["--motivate-worklist-length"] = b(o.motivate_worklist_length);
  h["--num-state-per-group"] = i(o.num_state_per_group);
  h["--group-num"] = i(o.group_num);
  h["--tuning"] = b(o.tuning);
  h["--pc-use-uvm"] = b(o.pc_use_uvm);
  h["--adaptive-aas"] = b(o.adaptive_aas);
  h["--try-adaptive-aas"] = b(o.try_adaptive_aas);
  h["--compress-prec-table"] = b(o.compress_prec_table);
  h["--dump-reports"] = s(o.dump_reports);
  h["--window"] = i(o.window);
  h["--chunk"] = i(o.chunk);
  h["--tile-states"] = i(o.tile_states);
  h["--tile-mode"] = i(o.tile_mode);
  for (int k = 1; k < argc; k++) {
    std::string a = argv[k];
    if (a == "-h" || a == "-?" || a == "--help") {
      o.show_help = true;
      continue;
    }
    std::string name = a, val;
    bool has_val = false;
    size_t eq = a.find('=');
    if (a.rfind("--", 0) == 0 && eq != std::string::npos) {
      name = a.substr(0, eq);
      val = a.substr(eq + 1);
      has_val = true;
    }
    auto it = h.find(name);
    if (it == h.end()) {
      err = "Unrecognised token: " + a;
      return false;
    }
    if (!has_val) {
      if (k + 1 >= argc) {
        err = "Expected argument following " + name;
        return false;
      }
      val = argv[++k];
    }
    if (!it->second(val)) {
      err = "Unable to convert '" + val + "' for option " + name;
      return false;
    }
  }
  if (o.show_help) return true;  // help needs no input
  if (o.input_filename.empty()) {
    err = "Option --input is required";
    return false;
  }
  if (o.nfa_filename.empty()) {
    err = "Option --automata is required";
    return false;
  }
  return true;
}

void print_help() {
  std::cout << "usage: ngap -a <file.anml> -i <input> --algorithm <name> [options]\n"
               "algorithms: blockinggroups NAPgroups nonblockinggroups nonblockingr1groups\n"
               "            nonblockingr2groups nonblockingpcgroups nonblockingallgroups\n"
               "options: --input-start-pos --input-len --split-entire-inputstream-to-chunk-size\n"
               "         --duplicate-input-stream --group-num --unique --unique-frequency\n"
               "         --result-capacity --data-buffer-fetch-size --add-aan-start\n"
               "         --add-aas-interval --active-threshold --precompute-cutoff\n"
               "         --precompute-depth --compress-prec-table --adaptive-aas --tuning\n"
               "         --report-off --validation --quick-validation --max-nfa-size\n"
               "         --quit-degree --remove-degree --app-name --dump-reports <file>\n"
               "         --window --chunk --tile-states --tile-mode (0 auto, 1 shared, 2 global)\n";
}

std::string err_msg() {
  char buf[1024];
  ngap_last_error(buf, sizeof(buf));
  return buf;
}

int algo_id(const std::string& a) {
  if (a == "blockinggroups") return NGAP_ALGO_BLOCKING;
  if (a == "NAPgroups") return NGAP_ALGO_NAP;
  if (a == "nonblockinggroups") return NGAP_ALGO_NONBLOCKING;
  if (a == "nonblockingr1groups") return NGAP_ALGO_NONBLOCKING_R1;
  if (a == "nonblockingr2groups") return NGAP_ALGO_NONBLOCKING_R2;
  if (a == "nonblockingpcgroups") return NGAP_ALGO_NONBLOCKING_PC;
  if (a == "nonblockingallgroups") return NGAP_ALGO_NONBLOCKING_ALL;
  return -1;
}

void print_vector(const std::vector<uint64_t>& v) {
  size_t n = std::min<size_t>(v.size(), 40);
  for (size_t i = 0; i < n; i++) printf("0x%lx, ", (unsigned long)v[i]);
  printf(v.size() > 40 ? "...\n" : "\n");
}

// --dump-reports: the sorted unique reports as raw little-endian u64; false,
// with a message on stderr, when the file cannot be written in full.
bool dump_reports(const std::string& path, const std::vector<uint64_t>& v) {
  FILE* df = fopen(path.c_str(), "wb");
  if (!df) {
    std::cerr << "Error: cannot open " << path << " for writing" << std::endl;
    return false;
  }
  const size_t n = v.empty() ? 0 : fwrite(v.data(), sizeof(uint64_t), v.size(), df);
  const bool closed = fclose(df) == 0;
  if (n != v.size() || !closed) {
    std::cerr << "Error: writing " << path << " failed" << std::endl;
    return false;
  }
  return true;
}

// --tuning (ngap.cu:1995-2056): the reference reruns the whole input over a
// grid of its knobs (fetch size x AAS interval x active threshold) and keeps
// the fastest run that validates. The knobs here are the engine's: window,
// chunk length and, for the privatizing algorithms, the active threshold. A
// candidate counts only when its reports equal the first candidate's. The
// best choice is written back into mp for the run that follows.
bool tune(ngap_engine* eng, const ngap_tables* tables, const std::vector<uint8_t>& ss,
          uint64_t total, ngap_match_params& mp) {
  const bool priv = mp.algorithm == NGAP_ALGO_NONBLOCKING_R1 ||
                    mp.algorithm == NGAP_ALGO_NONBLOCKING_R2 ||
                    mp.algorithm == NGAP_ALGO_NONBLOCKING_ALL;
  const std::vector<int> windows{256, 512, 1024, 2048, 4096};
  const std::vector<int> chunks{0, 4096, 16384};
  const std::vector<int> thresholds =
      priv ? std::vector<int>{0, 8, 16, 24, 32} : std::vector<int>{mp.active_threshold};
  std::vector<uint64_t> base;
  bool have_base = false;
  double best_thr = -1;
  int best[3] = {mp.window, mp.chunk, mp.active_threshold};
  const auto t_all = std::chrono::steady_clock::now();
  for (int w : windows)
    for (int th : thresholds)
      for (int ch : chunks) {
        const auto t0 = std::chrono::steady_clock::now();
        printf("[Tuning] Try choice: \n   window=%d, chunk=%d, active_threshold=%d\n", w, ch, th);
        ngap_match_params m = mp;
        m.window = w;
        m.chunk = ch;
        m.active_threshold = th;
        int rc = ngap_match(eng, tables, ss.data(), 0, &m, nullptr);
        if (rc == NGAP_OK) rc = ngap_engine_sync(eng);
        bool pass = rc == NGAP_OK;
        double thr = -1;
        if (pass) {
          float a = 0, b = 0;
          ngap_last_times_ms(eng, &a, &b);
          thr = (double)total / (((double)a + (double)b) * 1000.0);
          if (!m.report_off) {
            uint64_t raw = 0, uniq = 0;
            ngap_results_count(eng, &raw, &uniq);
            std::vector<uint64_t> res(uniq);
            if (uniq) ngap_results_copy(eng, res.data(), uniq);
            if (!have_base) {
              base.swap(res);
              have_base = true;
            } else {
              pass = res == base;
            }
          }
        }
        if (pass && thr > best_thr) {
          best_thr = thr;
          best[0] = w;
          best[1] = ch;
          best[2] = th;
          printf("[Tuning] Update best choice: \n   window=%d, chunk=%d, active_threshold=%d "
                 "max_throughput=%f\n", best[0], best[1], best[2], best_thr);
        } else {
          printf("[Tuning] Keep best choice: \n   window=%d, chunk=%d, active_threshold=%d "
                 "max_throughput=%f\n", best[0], best[1], best[2], best_thr);
        }
        const double sec =
            std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        std::cout << "[Tuning] " << sec << " seconds\n";
      }
  const double all =
      std::chrono::duration<double>(std::chrono::steady_clock::now() - t_all).count();
  std::cout << "[Tuning] Total time: " << all << " seconds\n";
  if (best_thr < 0) {
    std::cout << "ERROR: no tuning choice ran: " << err_msg() << std::endl;
    return false;
  }
  printf("[Tuning] Tuning completed: the best choice is\n   window=%d, chunk=%d, "
         "active_threshold=%d\n", best[0], best[1], best[2]);
  mp.window = best[0];
  mp.chunk = best[1];
  mp.active_threshold = best[2];
  return true;
}

// --motivate-worklist-length (ngap.cu:1843-1866): the reference appends the
// worklist length fetched per round to a file named after --app-name. The
// engine has no global rounds; it records each unit's worklist work (entries
// expanded plus entries injected by the warp that matched one tile over one
// chunk of a segment), written one unit per line: segment, tile, first and
// last position (relative to the segment), work.
bool save_worklist(ngap_engine* eng, const std::string& app_name) {
  int64_t n = 0;
  if (ngap_trace_copy(eng, nullptr, 0, &n) != NGAP_OK) {
    std::cout << "ERROR: " << err_msg() << std::endl;
    return false;
  }
  std::vector<ngap_unit_trace> tr((size_t)std::max<int64_t>(n, 1));
  if (n > 0 && ngap_trace_copy(eng, tr.data(), n, &n) != NGAP_OK) {
    std::cout << "ERROR: " << err_msg() << std::endl;
    return false;
  }
  const std::string path = (app_name.empty() ? std::string("ngap") : app_name) + ".worklist.txt";
  printf("Save froniter length file to %s\n", path.c_str());
  FILE* f = fopen(path.c_str(), "w");
  if (!f) {
    std::cerr << "Error: cannot open " << path << " for writing" << std::endl;
    return false;
  }
  for (int64_t i = 0; i < n; i++)
    fprintf(f, "%d %d %lld %lld %llu\n", tr[i].stream, tr[i].tile, (long long)tr[i].lo,
            (long long)tr[i].hi, (unsigned long long)tr[i].work);
  if (fclose(f) != 0) {
    std::cerr << "Error: writing " << path << " failed" << std::endl;
    return false;
  }
  return true;
}

}  // namespace

int main(int argc, char** argv) {
  printf("Command: ");
  for (int i = 0; i < argc; i++) printf("%s ", argv[i]);
  printf("\n");
  Options o;
  std::string perr;
  if (!parse_args(argc, argv, o, perr)) {
    std::cerr << "Error in command line: " << perr << std::endl;
    return 1;
  }
  if (o.show_help) {
    print_help();
    return 0;
  }

  // input stream (SymbolStream::readFromFile + slice, main.cu:45-50)
  std::ifstream f(o.input_filename, std::ios::binary);
  if (!f) {
    std::cout << " Error: no such input file." << std::endl;
    return 255;
  }
  std::vector<uint8_t> old_ss((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
  std::cout << "read input stream from file = " << o.input_filename << std::endl;
  std::cout << "input_stream_size = " << old_ss.size() << std::endl;
  if (o.input_start_pos != -1 && o.input_len != -1) {
    size_t st = (size_t)std::max(o.input_start_pos, 0);
    size_t len = (size_t)std::max(o.input_len, 0);
    if (st > old_ss.size()) st = old_ss.size();
    if (st + len > old_ss.size()) {
      len = old_ss.size() - st;
      std::cout << "the input is shorter than the length specified, just slice to end" << std::endl;
    }
    old_ss = std::vector<uint8_t>(old_ss.begin() + st, old_ss.begin() + st + len);
  }

  ngap_nfa* nfa = nullptr;
  if (ngap_nfa_load_anml(o.nfa_filename.c_str(), &nfa) != NGAP_OK) {
    std::cout << err_msg() << std::endl;
    return 255;
  }
  std::cout << "load automata from file = " << o.nfa_filename << std::endl;
  std::cout << "NFA Info:\n    total_state_number = " << ngap_nfa_num_states(nfa) << std::endl;

  ngap_group_opts go{o.group_num, o.max_nfa_size, o.quit_degree ? 1 : 0, o.remove_degree ? 1 : 0};
  ngap_groups* groups = nullptr;
  if (ngap_groups_build(nfa, &go, &groups) != NGAP_OK) {
    std::cout << err_msg() << std::endl;
    return 255;
  }
  int64_t cc_total = 0, cc_failed = 0, cc_big = 0;
  ngap_groups_cc_stats(groups, &cc_total, &cc_failed, &cc_big);
  printf("limit_out_degree_on_ccs: num_succeed %lld, num_fail %lld\n",
         (long long)(cc_total - cc_failed), (long long)cc_failed);
  const int group_num = ngap_groups_count(groups);
  if (group_num < o.group_num)
    printf("warning: cc_num is less than group_num = %d, new group_num will be %d\n", o.group_num,
           group_num);

  // duplicate + segment (main.cu:81-102)
  std::vector<uint8_t> ss;
  for (int d = 0; d < o.duplicate_input_stream; d++) ss.insert(ss.end(), old_ss.begin(), old_ss.end());
  int64_t seg_len = o.split_chunk_size > 0 ? o.split_chunk_size : (int64_t)ss.size();
  int64_t num_seg = seg_len > 0 ? (int64_t)ss.size() / seg_len : 0;
  printf("grouped_nfas.size = %d pl.num_seg=%lld\n", group_num, (long long)num_seg);
  std::cout << "Input Stream Info:\n    input_start_pos = " << o.input_start_pos
            << "\n    input_length = " << o.input_len
            << "\n    split_entire_inputstream_to_chunk_size = " << o.split_chunk_size
            << "\n    dup_input_stream = " << o.duplicate_input_stream << std::endl;
  const int algo = algo_id(o.algorithm);
  if (algo < 0) {
    std::cout << "not supported algoritm " << o.algorithm << std::endl;
    printf("FINISHED!\n");
    return 0;
  }
  if (algo == NGAP_ALGO_NAP && o.add_aas_start > 0) {  // ngap.cu:308-312
    printf("add_aas_start should be set to 0\n");
    return 255;
  }
  if (num_seg <= 0) {
    printf("input is empty after segmentation\n");
    return 255;
  }
  const bool is_dup = o.duplicate_input_stream > 1 &&
                      (o.split_chunk_size == -1 || o.split_chunk_size == o.input_len);

  ngap_table_opts to{};
  to.device = 0;
  to.precompute_depth = o.precompute_depth;
  to.precompute_cutoff = o.precompute_cutoff;
  to.tile_states = o.tile_states;
  to.tile_mode = o.tile_mode;
  ngap_tables* tables = nullptr;
  ngap_engine* eng = nullptr;
  if (ngap_tables_build(groups, &to, &tables) != NGAP_OK || ngap_engine_create(0, &eng) != NGAP_OK) {
    std::cout << err_msg() << std::endl;
    return 255;
  }
  ngap_match_params mp{};
  mp.algorithm = algo;
  mp.num_seg = num_seg;
  mp.seg_len = seg_len;
  mp.is_dup = is_dup ? 1 : 0;
  mp.unique = o.unique ? 1 : 0;
  mp.active_threshold = o.active_threshold;
  mp.report_off = o.report_off ? 1 : 0;
  mp.result_capacity = o.output_capacity;
  mp.window = o.window;
  mp.chunk = o.chunk;
  const uint64_t total = (uint64_t)num_seg * (uint64_t)seg_len;
  if (o.tuning && !tune(eng, tables, ss, total, mp)) return 255;
  if (o.motivate_worklist_length) ngap_engine_set_trace(eng, 1);
  int rc = ngap_match(eng, tables, ss.data(), 0, &mp, nullptr);
  if (rc == NGAP_OK) rc = ngap_engine_sync(eng);
  if (rc != NGAP_OK && rc != NGAP_E_OVERFLOW_RESULTS) {
    std::cout << "ERROR: " << err_msg() << std::endl;
    return 255;
  }
  if (o.motivate_worklist_length && !save_worklist(eng, o.app_name)) return 255;
  float match_ms = 0, sort_ms = 0;
  ngap_last_times_ms(eng, &match_ms, &sort_ms);
  const double ms = (double)match_ms + (double)sort_ms;
  const double thr = (double)total / (ms * 1000.0);
  uint64_t raw = 0, uniq = 0;
  ngap_results_count(eng, &raw, &uniq);
  const bool blocking = algo == NGAP_ALGO_BLOCKING;
  if (blocking)
    std::cout << "ngap elapsed time: " << ms / 1000.0 << " seconds, throughput = " << thr << " MB/s "
              << std::endl;
  std::cout << "Results number: " << raw << std::endl;
  bool pass = true, dump_ok = true;
  if (o.validation) {
    const unsigned long long dupnum = o.duplicate_input_stream > 1 ? o.duplicate_input_stream : 1;
    if (o.report_off) {
      unsigned long long vn = (unsigned long long)o.quick_validation * dupnum;
      pass = o.quick_validation >= 0 && vn <= raw;
      printf(pass ? "Quick Validation PASS! (report off)\n" : "Quick Validation FAILED! (report off)\n");
    } else {
      std::vector<uint64_t> res(uniq);
      if (uniq) ngap_results_copy(eng, res.data(), uniq);
      std::cout << "Unique results number: " << res.size() << std::endl;
      printf("validation start.\n");
      if (o.quick_validation >= 0) {
        pass = (unsigned long long)o.quick_validation * dupnum == res.size();
        printf(pass ? "Quick Validation PASS!\n" : "Quick Validation FAILED!\n");
      } else {
        std::vector<uint64_t> ref(std::max<uint64_t>(raw + 16, 1024));
        double cpu_ms = 0;
        int64_t nref = ngap_cpu_validate_reference(groups, ss.data(), num_seg, seg_len, is_dup,
                                                   ref.data(), (int64_t)ref.size(), &cpu_ms);
        while (nref < 0) {
          ref.resize(ref.size() * 4);
          nref = ngap_cpu_validate_reference(groups, ss.data(), num_seg, seg_len, is_dup,
                                             ref.data(), (int64_t)ref.size(), &cpu_ms);
        }
        ref.resize((size_t)nref);
        std::cout << "Reference CPU elapsed time: " << (long long)cpu_ms << " ms, "
                  << (double)total / (cpu_ms * 1000.0) << " MB/s" << std::endl;
        printf("\n############ Validate result ############ \n");
        pass = ref == res;
        if (pass) printf("Validation PASS!\n");
        else printf("Validation FAILED!\n");
        printf("Result(%zu): \n", res.size());
        print_vector(res);
        printf("Reference result(%zu): \n", ref.size());
        print_vector(ref);
        printf("\n");
      }
      if (!o.dump_reports.empty()) dump_ok = dump_reports(o.dump_reports, res);
    }
  } else if (!o.dump_reports.empty() && !o.report_off) {
    std::vector<uint64_t> res(uniq);
    if (uniq) ngap_results_copy(eng, res.data(), uniq);
    dump_ok = dump_reports(o.dump_reports, res);
  }
  if (!blocking) {
    if (pass)
      std::cout << "ngap elapsed time: " << ms / 1000.0 << " seconds, throughput = " << thr
                << " MB/s " << std::endl;
    else
      std::cout << "ngap elapsed time: " << ms / 1000.0 << " seconds, WRONGTHRPUT(" << thr
                << ") MB/s " << std::endl;
  }
  if (rc == NGAP_E_OVERFLOW_RESULTS) std::cout << "WARNING: " << err_msg() << std::endl;
  ngap_engine_destroy(eng);
  ngap_tables_destroy(tables);
  ngap_groups_destroy(groups);
  ngap_nfa_destroy(nfa);
  printf("FINISHED!\n");
  return dump_ok ? 0 : 255;
}
