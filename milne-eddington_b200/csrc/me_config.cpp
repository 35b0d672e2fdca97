// me_config.cpp -- control-file reader with the reference's keyword semantics.
//
// Follows RDINPUT / Get_Keys (Src/RINPUT.c:361-563, 48-357) and the line
// reader STR_READ_LINE (Src/STR.c:387-460):
//   * a line whose first non-blank character is '#', '!' or '*' is a comment;
//     an inline '!' ends the line;
//   * `key = value`: the key is the text before the first '=', right-trimmed
//     and compared case-sensitively; keys shorter than 2 characters are
//     skipped; unknown keys are ignored; a repeated key overwrites;
//   * `lines` may repeat up to 20 times (Src/RINPUT.c:483-495);
//   * numbers are read with atoi/atof/sscanf and the same formats;
//   * YES/NO flags are case-insensitive and exact ("YES");
//   * Bounds_Btheta / Bounds_Bphi and the theta/phi regularisation targets
//     are in units of pi in the file and stored in radians.
// Errors the reference turns into exit() become ME_ERR_CONFIG here.
#include <ctype.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <strings.h>

#include <string>
#include <vector>

#include "../../include/me_b200.h"

namespace {

const double kPi = 3.14159265358979323846;

enum Key {
  K_LINES, K_VERBOSE, K_NUM_ITER, K_NUM_RUN, K_CONVG, K_CHISQ, K_DATA, K_WAV, K_WEIGHTS,
  K_SOLBOX, K_OUTFIT, K_CACHEPATH, K_RESULT, K_FITPATH, K_DAMP, K_ACCEPT, K_REJECT, K_LIMITS,
  K_B_BMOD, K_B_THETA, K_B_PHI, K_B_VLOS, K_B_DOPP, K_B_DAMP, K_B_ETA, K_B_CONT, K_B_BETA,
  K_F_BMOD, K_F_THETA, K_F_PHI, K_F_VLOS, K_F_DOPP, K_F_DAMP, K_F_ETA, K_F_CONT, K_F_BETA,
  K_R_BMOD, K_R_THETA, K_R_PHI, K_R_VLOS, K_R_DOPP, K_R_DAMP, K_R_ETA, K_R_CONT, K_R_BETA,
  K_VCOEF, K_LCOEF, K_ICRIT, K_SVDTHR, K_HMIREF, K_CACHEPROF, K_NTHREADS, K_NFIG, K_STEP,
  K_NPROF, K_CACHEINV,
  // keywords of this library
  K_PRECISION, K_RNGSEED, K_FILTER,
  K_COUNT
};

struct KeyDef {
  const char *name;
  const char *dflt;  // nullptr = required
};

// The reference's keyword table with its defaults (Src/RINPUT.c:400-458).
const KeyDef kKeys[K_COUNT] = {
    {"lines", nullptr},
    {"verbose", "1"},
    {"num_iter", "60"},
    {"num_run", "4"},
    {"convg_criteria", "1e-3"},
    {"chisq_criteria", "1.0"},
    {"data_path", nullptr},
    {"wavelength_path", nullptr},
    {"weights", "1., 1., 1., 1."},
    {"sol_box", "-1, -1, -1, -1"},
    {"output_fit", "NO"},
    {"cache_path", "./cache"},
    {"result_path", "./res.fits"},
    {"fit_path", "./fit.fits"},
    {"damp", "1e-3"},
    {"lambda_accept", "5.0"},
    {"lambda_reject", "5.0"},
    {"lambda_limits", "1e-5, 1e3"},
    {"Bounds_Bmod", "5, 6000"},
    {"Bounds_Btheta", "0, 1"},
    {"Bounds_Bphi", "0, 1"},
    {"Bounds_Vlos", "-20., 20."},
    {"Bounds_Dopp", "10, 80"},
    {"Bounds_Damp", "0.4, 0.8"},
    {"Bounds_Eta", "2, 90"},
    {"Bounds_Continuum", "0, 1e6"},
    {"Bounds_Beta", "0.1, 0.85"},
    {"Bmod_fixed", "NO"},
    {"Btheta_fixed", "NO"},
    {"Bphi_fixed", "NO"},
    {"Vlos_fixed", "NO"},
    {"Dopp_fixed", "NO"},
    {"Damp_fixed", "NO"},
    {"Eta_fixed", "NO"},
    {"Continuum_fixed", "NO"},
    {"Beta_fixed", "NO"},
    {"Bmod_Regularization", "NO"},
    {"Btheta_Regularization", "YES, 0.5, 1e-4"},
    {"Bphi_Regularization", "NO"},
    {"Vlos_Regularization", "NO"},
    {"Dopp_Regularization", "NO, 20, 0.05"},
    {"Damp_Regularization", "NO, 0.5, 80"},
    {"Eta_Regularization", "NO, 2.0, 0.01"},
    {"Continuum_Regularization", "NO"},
    {"Beta_Regularization", "NO"},
    {"VCoeffi", "100."},
    {"LCoeffi", "250."},
    {"Icriteria", "100."},
    {"SVDthreshold", "1e-6"},
    {"HMI_REF", "No"},
    {"Cache_prof", "No"},
    {"Nthreads", "4"},
    {"Nfigures", "6"},
    {"Step", "1000., 2., 2., 2., 20., 0.3, 30., 1e5, 0.3"},
    {"nprofiles", "20"},
    {"Cache_inv", "No"},
    {"precision", "FP32"},
    {"rng_seed", "0"},
    {"filter", "0"},
};

const size_t kKeyLen = 64;    // Src/STR.h:14
const size_t kLineLen = 512;  // Src/STR.h:15

void trim(std::string &s) {
  size_t a = 0;
  while (a < s.size() && isspace((unsigned char)s[a])) a++;
  size_t b = s.size();
  while (b > a && isspace((unsigned char)s[b - 1])) b--;
  s = s.substr(a, b - a);
}

std::string upper(std::string s) {
  for (auto &c : s) c = (char)toupper((unsigned char)c);
  return s;
}

bool is_yes(const std::string &v) { return strcasecmp(v.c_str(), "YES") == 0; }

void set_err(char *buf, size_t len, const std::string &msg) {
  if (buf && len) snprintf(buf, len, "%s", msg.c_str());
}

struct Parsed {
  std::string val[K_COUNT];
  bool set[K_COUNT] = {};
  std::vector<std::string> lines;
};

// STR_READ_LINE + the key/value split of RDINPUT (Src/RINPUT.c:465-545).
int scan(const char *text, Parsed &P, char *err, size_t errlen) {
  for (int k = 0; k < K_COUNT; k++)
    if (kKeys[k].dflt) P.val[k] = kKeys[k].dflt;
  const char *p = text;
  while (*p) {
    const char *e = strchr(p, '\n');
    std::string line = e ? std::string(p, e - p) : std::string(p);
    p = e ? e + 1 : p + line.size();
    // leading blanks, comment lines
    size_t a = 0;
    while (a < line.size() && isspace((unsigned char)line[a])) a++;
    line = line.substr(a);
    if (line.empty() || line[0] == '#' || line[0] == '!' || line[0] == '*') continue;
    size_t bang = line.find('!');
    if (bang != std::string::npos) line = line.substr(0, bang);
    while (!line.empty() && isspace((unsigned char)line.back())) line.pop_back();
    size_t eq = line.find('=');
    if (eq == std::string::npos || eq <= 1) continue;
    if (eq > kKeyLen - 1) continue;  // "keyword too long": skipped with a warning
    std::string key = line.substr(0, eq);
    while (!key.empty() && isspace((unsigned char)key.back())) key.pop_back();
    std::string value = line.substr(eq + 1);
    size_t v0 = 0;
    while (v0 < value.size() && isspace((unsigned char)value[v0])) v0++;
    value = value.substr(v0);
    if (value.size() > kLineLen - 1) value.resize(kLineLen - 1);
    if (key == kKeys[K_LINES].name) {
      P.lines.push_back(value);
      P.set[K_LINES] = true;
      if (P.lines.size() > (size_t)ME_MAX_LINES) {
        set_err(err, errlen, "keyword lines given more than 20 times");
        return ME_ERR_CONFIG;
      }
      continue;
    }
    for (int k = 1; k < K_COUNT; k++) {
      if (key == kKeys[k].name) {
        std::string v = value;
        trim(v);
        P.val[k] = v;
        P.set[k] = true;
        break;
      }
    }
  }
  return ME_OK;
}

int read_pair(const std::string &s, double *a, double *b) {
  return sscanf(s.c_str(), "%lf, %lf", a, b);
}

// Get_Keys (Src/RINPUT.c:48-357).
int convert(const Parsed &P, me_config *c, char *err, size_t errlen) {
  for (int k = 0; k < K_COUNT; k++) {
    if (!kKeys[k].dflt && !P.set[k]) {
      set_err(err, errlen, std::string("required keyword missing: ") + kKeys[k].name);
      return ME_ERR_CONFIG;
    }
  }
  c->verbose = atoi(P.val[K_VERBOSE].c_str());
  c->nline = (int)P.lines.size();
  for (int i = 0; i < c->nline; i++) {
    if (sscanf(P.lines[i].c_str(), "%lf, %lf", &c->line_lambda0[i], &c->line_geff[i]) != 2) {
      set_err(err, errlen, "error in reading the spectral line info: " + P.lines[i]);
      return ME_ERR_CONFIG;
    }
  }
  c->lines_seen = P.set[K_LINES];
  c->num_iter = atoi(P.val[K_NUM_ITER].c_str());
  c->num_run = atoi(P.val[K_NUM_RUN].c_str());
  c->convg_criteria = atof(P.val[K_CONVG].c_str());
  c->chisq_criteria = atof(P.val[K_CHISQ].c_str());
  snprintf(c->data_path, sizeof(c->data_path), "%s", P.val[K_DATA].c_str());
  snprintf(c->wavelength_path, sizeof(c->wavelength_path), "%s", P.val[K_WAV].c_str());
  c->data_path_seen = P.set[K_DATA];
  c->wavelength_path_seen = P.set[K_WAV];
  if (sscanf(P.val[K_WEIGHTS].c_str(), "%lf, %lf, %lf, %lf", &c->weights[0], &c->weights[1],
             &c->weights[2], &c->weights[3]) != 4) {
    set_err(err, errlen, "4 floats needed for weights");
    return ME_ERR_CONFIG;
  }
  if (sscanf(P.val[K_SOLBOX].c_str(), "%d, %d, %d, %d", &c->sol_box[0], &c->sol_box[1],
             &c->sol_box[2], &c->sol_box[3]) != 4) {
    set_err(err, errlen, "4 integers needed for the sol_box");
    return ME_ERR_CONFIG;
  }
  c->output_fit = is_yes(P.val[K_OUTFIT]);
  snprintf(c->cache_path, sizeof(c->cache_path), "%s", P.val[K_CACHEPATH].c_str());
  snprintf(c->result_path, sizeof(c->result_path), "%s", P.val[K_RESULT].c_str());
  snprintf(c->fit_path, sizeof(c->fit_path), "%s", P.val[K_FITPATH].c_str());
  c->damp = atof(P.val[K_DAMP].c_str());
  c->lambda_accept = atof(P.val[K_ACCEPT].c_str());
  c->lambda_reject = atof(P.val[K_REJECT].c_str());
  int nread = read_pair(P.val[K_LIMITS], &c->lambda_limits[0], &c->lambda_limits[1]);
  if (c->lambda_accept < 1.5 || c->lambda_reject < 1.5) {
    set_err(err, errlen, "lambda_accept and lambda_reject should be larger than 1.5");
    return ME_ERR_CONFIG;
  }
  if (nread != 2) {
    set_err(err, errlen, "2 floats needed for the lambda limits");
    return ME_ERR_CONFIG;
  }
  for (int i = 0; i < 9; i++) {
    if (read_pair(P.val[K_B_BMOD + i], &c->bounds[i][0], &c->bounds[i][1]) != 2) {
      set_err(err, errlen, std::string("error reading two doubles for key ") + kKeys[K_B_BMOD + i].name);
      return ME_ERR_CONFIG;
    }
    if (i == 1 || i == 2) {
      c->bounds[i][0] *= kPi;
      c->bounds[i][1] *= kPi;
    }
  }
  c->regul_any = 0;
  for (int i = 0; i < 9; i++) {
    c->fixed[i] = is_yes(P.val[K_F_BMOD + i]);
    char head[kKeyLen];
    double v = 0, w = 0;
    c->regul[i] = 0;
    c->regul_value[i] = 0;
    c->regul_weight[i] = 0;
    int n = sscanf(P.val[K_R_BMOD + i].c_str(), "%63[^,], %lf, %lf", head, &v, &w);
    if (n == 3) {
      std::string h = head;
      trim(h);
      if (is_yes(upper(h))) {
        c->regul[i] = 1;
        c->regul_any = 1;
        c->regul_value[i] = (i == 1 || i == 2) ? v * kPi : v;
        c->regul_weight[i] = w;
      } else {
        c->regul_value[i] = v;
        c->regul_weight[i] = w;
      }
    }
  }
  c->vcoeffi = atof(P.val[K_VCOEF].c_str());
  c->lcoeffi = atof(P.val[K_LCOEF].c_str());
  c->icriteria = atof(P.val[K_ICRIT].c_str());
  c->svd_threshold = atof(P.val[K_SVDTHR].c_str());
  c->hmi_ref = is_yes(P.val[K_HMIREF]);
  c->cache_prof = is_yes(P.val[K_CACHEPROF]);
  if (c->cache_prof) c->output_fit = 0;  // Src/RINPUT.c:318
  c->cache_inv = is_yes(P.val[K_CACHEINV]);
  c->nthreads = atoi(P.val[K_NTHREADS].c_str());
  c->nfigures = atoi(P.val[K_NFIG].c_str());
  if (sscanf(P.val[K_STEP].c_str(), "%lf, %lf, %lf, %lf, %lf, %lf, %lf, %lf, %lf", &c->step[0],
             &c->step[1], &c->step[2], &c->step[3], &c->step[4], &c->step[5], &c->step[6],
             &c->step[7], &c->step[8]) != 9) {
    set_err(err, errlen, "9 floats needed for the steps");
    return ME_ERR_CONFIG;
  }
  c->nprofiles = atoi(P.val[K_NPROF].c_str());
  std::string prec = upper(P.val[K_PRECISION]);
  if (prec == "FP32")
    c->precision = ME_PREC_FP32;
  else if (prec == "FP64")
    c->precision = ME_PREC_FP64;
  else {
    set_err(err, errlen, "precision must be FP32 or FP64");
    return ME_ERR_CONFIG;
  }
  c->rng_seed = strtoull(P.val[K_RNGSEED].c_str(), nullptr, 0);
  // filter = FWHM [mA], points: a Gaussian instrument filter (not in the
  // reference); "0" = none
  c->filter_fwhm = 0.0;
  c->filter_points = 1;
  {
    double fw = 0.0;
    int np = 0;
    const int got = sscanf(P.val[K_FILTER].c_str(), "%lf, %d", &fw, &np);
    if (got >= 1 && fw > 0.0) {
      if (got != 2 || np < 1 || np > ME_MAX_FILTER || np % 2 == 0) {
        set_err(err, errlen, "filter needs FWHM [mA] and an odd number of points up to 63");
        return ME_ERR_CONFIG;
      }
      c->filter_fwhm = fw;
      c->filter_points = np;
    } else if (got < 1 || fw < 0.0) {
      set_err(err, errlen, "filter must be 0 or `FWHM, points`");
      return ME_ERR_CONFIG;
    }
  }
  // Nfigures selects a row of the region table (Src/FADDEEVA.c:471-477);
  // rows exist for Nfigures <= 8 only.
  if (c->nfigures > 8) {
    set_err(err, errlen, "Nfigures above 8 has no accuracy row");
    return ME_ERR_CONFIG;
  }
  return ME_OK;
}

}  // namespace

extern "C" int me_config_init(me_config *cfg) {
  if (!cfg) return ME_ERR_ARG;
  memset(cfg, 0, sizeof(*cfg));
  Parsed P;
  scan("", P, nullptr, 0);
  // the defaults table has no `lines` / paths; convert() with them present
  P.set[K_LINES] = P.set[K_DATA] = P.set[K_WAV] = true;
  int rc = convert(P, cfg, nullptr, 0);
  cfg->lines_seen = cfg->data_path_seen = cfg->wavelength_path_seen = 0;
  return rc;
}

extern "C" int me_config_parse_text(const char *text, me_config *cfg, char *err, size_t errlen) {
  if (!text || !cfg) return ME_ERR_ARG;
  memset(cfg, 0, sizeof(*cfg));
  Parsed P;
  int rc = scan(text, P, err, errlen);
  if (rc) return rc;
  return convert(P, cfg, err, errlen);
}

extern "C" int me_config_parse(const char *path, me_config *cfg, char *err, size_t errlen) {
  if (!path || !cfg) return ME_ERR_ARG;
  FILE *f = fopen(path, "rb");
  if (!f) {
    set_err(err, errlen, std::string("cannot open control file: ") + path);
    return ME_ERR_IO;
  }
  std::string text;
  char buf[4096];
  size_t n;
  while ((n = fread(buf, 1, sizeof(buf), f)) > 0) text.append(buf, n);
  fclose(f);
  return me_config_parse_text(text.c_str(), cfg, err, errlen);
}
