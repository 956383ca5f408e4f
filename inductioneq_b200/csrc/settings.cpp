// settings.cpp -- parsing of the reference's "-DKEY=VAL" settings string and kernel path
// list (matlab/generate_settings.m:3-33, compute_numerical_solution_setup.m:57-137), and
// expansion of the compact SBP coefficient tables.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <sstream>

#include "ieq_host.h"

namespace ieq {

struct SbpTableSource {
  int nb, width, sign, explicit_rows;
  const double *rows;
};
struct SbpOperatorSource {
  int order, extended, nb, sw, w_hod;
  SbpTableSource D, Dadj, DHO;
  const double *minv;
  SbpTableSource lap[3];
};

#include "sbp_tables.inc"

static const char *kTestcases[] = {"rotation_2D",     "rotation_3D",        "hall_periodic",
                                   "hall_travelling_wave", "confined_domain", "alfven_periodic_2D",
                                   "rotation_gaussian", "hall_circular_wave"};

static const char *kIntegrators[] = {"SSPRK33", "SSPRK104", "KennedyCarpenterLewis2R54C",
                                     "CalvoFrancoRandez2R64", "CarpenterKennedy2N54",
                                     "ToulorgeDesmet2N84F"};

int integrator_id(const std::string &name) {
  for (int i = 0; i < 6; ++i)
    if (name == kIntegrators[i]) return i;
  return -1;
}

static std::string basename_of(const std::string &p) {
  size_t k = p.find_last_of("/\\");
  return k == std::string::npos ? p : p.substr(k + 1);
}

static bool parse_double(const std::string &v, double &out) {
  char *end = nullptr;
  out = std::strtod(v.c_str(), &end);
  return end && *end == '\0' && !v.empty();
}

bool parse_settings(const char *settings, const char *const *paths, int n_paths, Settings &s,
                    std::string &err) {
  std::istringstream in(settings ? settings : "");
  std::string tok;
  bool have_nodes[3] = {false, false, false};
  while (in >> tok) {
    if (tok.rfind("-D", 0) != 0) continue;   // OpenCL compiler options are ignored
    std::string kv = tok.substr(2), key = kv, val = "1";
    size_t eq = kv.find('=');
    if (eq != std::string::npos) {
      key = kv.substr(0, eq);
      val = kv.substr(eq + 1);
    }
    double x = 0;
    const char *axes[3] = {"X", "Y", "Z"};
    bool done = false;
    for (int a = 0; a < 3 && !done; ++a) {
      if (key == std::string("NODES_") + axes[a]) {
        if (!parse_double(val, x) || x < 1 || x != std::floor(x)) {
          err = "bad " + key;
          return false;
        }
        s.nodes[a] = (int)x;
        have_nodes[a] = true;
        done = true;
      } else if (key == std::string("D") + axes[a]) {
        if (!parse_double(val, x) || !(x > 0)) {
          err = "bad " + key;
          return false;
        }
        s.d[a] = x;
        s.have_d[a] = true;
        done = true;
      } else if (key == std::string(axes[a]) + "MIN") {
        if (!parse_double(val, s.xmin[a])) { err = "bad " + key; return false; }
        done = true;
      } else if (key == std::string(axes[a]) + "MAX") {
        if (!parse_double(val, s.xmax[a])) { err = "bad " + key; return false; }
        done = true;
      }
    }
    if (done) continue;
    if (key == "DT") {
      if (!parse_double(val, s.dt)) { err = "bad DT"; return false; }
    } else if (key == "REAL") {
      if (val == "float") s.real_float = true;
      else if (val == "double") s.real_float = false;
      else { err = "REAL must be float or double"; return false; }
    } else if (key == "W_SIZE") {
      if (!parse_double(val, x) || x < 1) { err = "bad W_SIZE"; return false; }
      s.w_size = (int)x;
    } else if (key == "HO_DISSIPATION_FACTOR") {
      parse_double(val, s.hod_factor);
    } else if (key == "MP2MIN") {
      parse_double(val, s.mp2min);
    } else if (key == "MP2MAX") {
      parse_double(val, s.mp2max);
    } else if (key == "CMIN") {
      parse_double(val, s.cmin);
    } else if (key == "CMAX") {
      parse_double(val, s.cmax);
    } else if (key == "BNODES") {
      if (!parse_double(val, x) || x < 0) { err = "bad BNODES"; return false; }
      s.bnodes = (int)x;
    } else if (key == "TC_OMEGA") {
      parse_double(val, s.omega);
    } else if (key == "IEQ_INTEGRATOR") {
      if (integrator_id(val) < 0) { err = "unknown time integrator " + val; return false; }
      s.integrator = val;
    } else if (key == "IEQ_VARIABLE_U") {
      s.variable_u = val != "0";
    } else if (key == "IEQ_STAGE_KERNEL") {
      if (val == "AUTO") s.stage_kernel = 0;
      else if (val == "COLUMN") s.stage_kernel = 1;
      else if (val == "NODE") s.stage_kernel = 2;
      else if (val == "BRICK") s.stage_kernel = 3;
      else if (val == "LIST") s.stage_kernel = 4;
      else if (val == "ZMARCH") s.stage_kernel = 5;
      else { err = "IEQ_STAGE_KERNEL must be AUTO, COLUMN, NODE, BRICK, LIST or ZMARCH"; return false; }
    } else if (key == "IEQ_COL_BLOCK" || key == "IEQ_CURL_BLOCK") {
      int *b = key == "IEQ_COL_BLOCK" ? s.col_block : s.curl_block;
      char tail = 0;
      if (std::sscanf(val.c_str(), "%dx%dx%d%c", &b[0], &b[1], &b[2], &tail) != 3 || b[0] < 1 || b[1] < 1 ||
          b[2] < 1 || b[0] * b[1] * b[2] != 128) {
        err = key + " must be XxYxZ with X * Y * Z = 128 (e.g. 32x4x1)";
        return false;
      }
    } else if (key == "IEQ_XBAND") {
      if (val != "0" && val != "1" && val != "2") {
        err = "IEQ_XBAND must be 0, 1 or 2";
        return false;
      }
      s.xband = std::atoi(val.c_str());
    } else if (key == "IEQ_ZMARCH_TZ") {
      char tail = 0;
      int v = 0;
      if (std::sscanf(val.c_str(), "%d%c", &v, &tail) != 1 || v < 0) {
        err = "IEQ_ZMARCH_TZ must be a non-negative integer (0: chosen per grid)";
        return false;
      }
      s.zmarch_tz = v;
    } else if (key == "IEQ_Z_OFFSET" || key == "IEQ_NZ_GLOBAL") {
      char tail = 0;
      int v = 0;
      if (std::sscanf(val.c_str(), "%d%c", &v, &tail) != 1 || (key == "IEQ_NZ_GLOBAL" && v < 0)) {
        err = key + " must be an integer (IEQ_NZ_GLOBAL >= 0)";
        return false;
      }
      (key == "IEQ_Z_OFFSET" ? s.zoff : s.nzg) = v;
    } else if (key == "IEQ_CG_LOOP") {
      if (val != "GRAPH" && val != "HOST") {
        err = "IEQ_CG_LOOP must be GRAPH or HOST";
        return false;
      }
      s.cg_host_loop = val == "HOST";
    } else if (key == "IEQ_CURL_Z") {
      if (val != "0" && val != "1" && val != "2") {
        err = "IEQ_CURL_Z must be 0, 1 or 2";
        return false;
      }
      s.curl_z = std::atoi(val.c_str());
    } else if (key == "IEQ_ADJOINT_PROGRAM") {
      if (val != "0" && val != "1") {
        err = "IEQ_ADJOINT_PROGRAM must be 0 or 1";
        return false;
      }
      s.adjoint_program = std::atoi(val.c_str());
    } else if (key == "IEQ_HODP") {
      if (val != "0" && val != "1") {
        err = "IEQ_HODP must be 0 or 1";
        return false;
      }
      s.hodp = std::atoi(val.c_str());
    } else if (key == "IEQ_CG_PASS_A") {
      if (val != "1" && val != "2") {
        err = "IEQ_CG_PASS_A must be 1 (per-node gather) or 2 (2.5D z march)";
        return false;
      }
      s.cg_passes = std::atoi(val.c_str());
    } else if (key == "IEQ_PDL") {
      if (val != "0" && val != "1") {
        err = "IEQ_PDL must be 0 or 1";
        return false;
      }
      s.pdl = val == "1";
    } else if (key == "IEQ_COL_PAIRS") {
      if (val != "0" && val != "1" && val != "4") {
        err = "IEQ_COL_PAIRS must be 0, 1 or 4";
        return false;
      }
      s.col_pairs = std::atoi(val.c_str());
    } else if (key == "USE_HALL") {
      s.hall = true;
    } else if (key == "USE_PERIODIC") {
      s.periodic = true;
    } else if (key == "USE_ARTIFICIAL_DISSIPATION") {
      s.dissipation = true;
    } else if (key == "USE_HIGH_ORDER_DISSIPATION") {
      s.diss_form = 1;
    } else if (key == "USE_FIRST_ORDER_DISSIPATION") {
      if (s.diss_form != 1) s.diss_form = 2;
    } else if (key == "USE_ADAPTIVE_DISSIPATION") {
      if (s.diss_form == 0) s.diss_form = 3;
    } else if (key == "USE_LAPLACE_WIDE_STENCIL_DIRICHLET") {
      s.laplace = 0;
    } else if (key == "USE_LAPLACE_NARROW_STENCIL_DIRICHLET") {
      s.laplace = 1;
    } else if (key == "USE_LAPLACE_WIDE_STENCIL_LNS") {
      s.laplace = 2;
    } else if (key == "REDUCE") {
      s.reduce = true;
    } else if (key.rfind("USE_UIBJ_", 0) == 0 || key.rfind("USE_SOURCE_", 0) == 0 ||
               key.rfind("USE_UJBI_", 0) == 0) {
      const std::string f = key.substr(key.rfind('_') + 1);
      int code = f == "CENTRAL" ? 0 : f == "SPLIT" ? 1 : f == "PRODUCT" ? 2 : f == "ZERO" ? 3 : -1;
      int *slot = key.rfind("USE_UIBJ_", 0) == 0 ? &s.uibj : key.rfind("USE_SOURCE_", 0) == 0 ? &s.source : &s.ujbi;
      const bool ok = (slot == &s.source) ? (code == 0 || code == 1 || code == 3) : (code >= 0 && code <= 2);
      if (!ok) { err = "unknown flux form " + key; return false; }
      *slot = code;
    }
    // REAL4, fp64_atomics and unknown keys are accepted as in an OpenCL build
  }
  // the kernel path list names the operator header and the testcase header
  for (int i = 0; i < n_paths; ++i) {
    if (!paths || !paths[i]) continue;
    const std::string b = basename_of(paths[i]);
    for (int o : {2, 4, 6}) {
      const std::string base = std::to_string(o) + (o == 2 ? "nd" : "th") + "Order";
      if (b == base + ".h") { s.order = o; s.extended = false; }
      if (b == base + "Extended.h") { s.order = o; s.extended = true; }
    }
    for (int t = 0; t < 8; ++t)
      if (b == std::string(kTestcases[t]) + ".h") s.testcase = t;
  }
  for (int a = 0; a < 3; ++a) {
    if (!have_nodes[a]) { err = "settings lack NODES_X/Y/Z"; return false; }
    if (!s.have_d[a]) {
      // initialize.m:12-21 computes D from the box when only the box is given
      const double span = s.xmax[a] - s.xmin[a];
      s.d[a] = s.periodic ? span / s.nodes[a] : span / (s.nodes[a] - 1.0);
      if (!(s.d[a] > 0)) { err = "settings lack DX/DY/DZ and a box"; return false; }
    }
  }
  if (s.order == 0) { err = "kernel path list lacks an operator header ({2,4,6}thOrder[Extended].h)"; return false; }
  if (s.testcase < 0) { err = "kernel path list lacks a known testcase header"; return false; }
  if (s.extended && s.laplace == 1) {
    err = "the narrow-stencil Laplacian is not derived for the extended operators";
    return false;
  }
  if (s.bnodes < 0) s.bnodes = s.laplace == 2 ? 0 : 1;   // initialize.m:105-114
  if (!s.dissipation) s.diss_form = 0;
  return true;
}

static SbpRows expand(const SbpTableSource &t) {
  SbpRows r;
  r.nb = t.nb;
  r.width = t.width;
  const int nrows = 2 * t.nb + 1;
  r.rows.assign((size_t)nrows * t.width, 0.0);
  if (t.explicit_rows) {
    for (int i = 0; i < nrows * t.width; ++i) r.rows[i] = t.rows[i];
    return r;
  }
  for (int j = 0; j <= t.nb; ++j)
    for (int c = 0; c < t.width; ++c) r.rows[(size_t)j * t.width + c] = t.rows[j * t.width + c];
  for (int j = 0; j < t.nb; ++j)
    for (int c = 0; c < t.width; ++c) {
      const double v = t.rows[j * t.width + (t.width - 1 - c)];
      r.rows[(size_t)(2 * t.nb - j) * t.width + c] = v == 0.0 ? 0.0 : t.sign * v;
    }
  return r;
}

bool load_operator(int order, bool extended, SbpOperator &op, std::string &err) {
  for (const SbpOperatorSource &src : kSbpOperators) {
    if (src.order != order || (src.extended != 0) != extended) continue;
    op.order = order;
    op.nb = src.nb;
    op.sw = src.sw;
    op.w_hod = src.w_hod;
    op.D = expand(src.D);
    op.Dadj = expand(src.Dadj);
    op.DHO = expand(src.DHO);
    op.minv.assign(2 * src.nb + 1, 0.0);
    for (int j = 0; j <= src.nb; ++j) op.minv[j] = op.minv[2 * src.nb - j] = src.minv[j];
    for (int l = 0; l < 3; ++l) {
      op.has_lap[l] = src.lap[l].rows != nullptr;
      if (op.has_lap[l]) op.lap[l] = expand(src.lap[l]);
    }
    return true;
  }
  err = "no operator of order " + std::to_string(order);
  return false;
}

}  // namespace ieq
