// Case files and output files in the reference's layouts (src/loquat_io.cu).
// The parameter file is the flat typed XML the reference reads with tinyxml2:
//   <parameters> <name type="int|scalar|model_mat|dimension|bool">value</name> ... </parameters>
// A small reader for exactly that shape is used here instead of a general XML library.
#include "rw_io.h"

#include <algorithm>
#include <charconv>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <numeric>
#include <sstream>
#include <thread>

namespace rw {

namespace {
// A real as an ostream prints it by default (printf's %g, six significant digits): the
// format of the reference's output writer.
inline void put_g(std::string& o, double v) {
  char buf[40];
  auto r = std::to_chars(buf, buf + sizeof(buf), v, std::chars_format::general, 6);
  o.append(buf, r.ptr);
}
inline void put_i(std::string& o, long long v) {
  char buf[24];
  auto r = std::to_chars(buf, buf + sizeof(buf), v);
  o.append(buf, r.ptr);
}
int io_threads() { return (int)std::max(1u, std::min(32u, std::thread::hardware_concurrency())); }
// Rows [0, n) formatted by fn(row, out) on several host threads, each into its own
// buffer, then written to f in order.
template <class Fn> bool put_rows(std::FILE* f, size_t n, size_t bytes_per_row, Fn fn) {
  const int nth = n < 8192 ? 1 : io_threads();
  std::vector<std::string> part(nth);
  auto run = [&](int t) {
    const size_t lo = n * t / nth, hi = n * (t + 1) / nth;
    part[t].reserve((hi - lo) * bytes_per_row);
    for (size_t q = lo; q < hi; ++q) fn(q, part[t]);
  };
  std::vector<std::thread> th;
  for (int t = 1; t < nth; ++t) th.emplace_back(run, t);
  run(0);
  for (auto& x : th) x.join();
  bool ok = true;
  for (auto& s : part) ok = ok && std::fwrite(s.data(), 1, s.size(), f) == s.size();
  return ok;
}
inline bool put_text(std::FILE* f, const std::string& s) { return std::fwrite(s.data(), 1, s.size(), f) == s.size(); }
}  // namespace

rw_case HostCase::view() const {
  rw_case c;
  c.params = params;
  c.codes = codes.data();
  c.pospres = pospres.data();
  c.velrhop = velrhop.data();
  c.idmassidx = idmassidx.data();
  c.stress = stress.data();
  c.strain = strain.data();
  c.normal = normal.empty() ? nullptr : normal.data();
  return c;
}

static std::string trim(const std::string& s) {
  size_t a = s.find_first_not_of(" \t\r\n"), b = s.find_last_not_of(" \t\r\n");
  return a == std::string::npos ? std::string() : s.substr(a, b - a + 1);
}

int read_xml_params(const std::string& path, std::map<std::string, std::pair<std::string, std::string>>* out,
                    std::string* msg) {
  std::ifstream f(path);
  if (!f) {
    *msg = "Cannot load the parameter file: " + path;
    return RW_ENOENT;
  }
  std::stringstream ss;
  ss << f.rdbuf();
  const std::string s = ss.str();
  size_t p = 0;
  // Skip declaration and comments; find the root element.
  auto skip_misc = [&]() {
    for (;;) {
      p = s.find('<', p);
      if (p == std::string::npos) return;
      if (s.compare(p, 2, "<?") == 0) {
        p = s.find("?>", p);
        if (p != std::string::npos) p += 2;
      } else if (s.compare(p, 4, "<!--") == 0) {
        p = s.find("-->", p);
        if (p != std::string::npos) p += 3;
      } else {
        return;
      }
    }
  };
  skip_misc();
  if (p == std::string::npos) {
    *msg = "no root element in " + path;
    return RW_EFORMAT;
  }
  size_t root_end = s.find('>', p);
  if (root_end == std::string::npos) {
    *msg = "unterminated root element in " + path;
    return RW_EFORMAT;
  }
  p = root_end + 1;
  for (;;) {
    skip_misc();
    if (p == std::string::npos) break;
    if (s.compare(p, 2, "</") == 0) break;  // end of root
    size_t gt = s.find('>', p);
    if (gt == std::string::npos) {
      *msg = "unterminated element in " + path;
      return RW_EFORMAT;
    }
    std::string head = s.substr(p + 1, gt - p - 1);
    bool selfclose = !head.empty() && head.back() == '/';
    if (selfclose) head.pop_back();
    size_t sp = head.find_first_of(" \t\r\n");
    std::string name = trim(head.substr(0, sp));
    std::string type;
    size_t tp = head.find("type");
    if (tp != std::string::npos) {
      size_t q1 = head.find('"', tp);
      size_t q2 = q1 == std::string::npos ? q1 : head.find('"', q1 + 1);
      if (q1 != std::string::npos && q2 != std::string::npos) type = head.substr(q1 + 1, q2 - q1 - 1);
    }
    std::string text;
    if (!selfclose) {
      std::string close = "</" + name + ">";
      size_t ce = s.find(close, gt + 1);
      if (ce == std::string::npos) {
        *msg = "missing " + close + " in " + path;
        return RW_EFORMAT;
      }
      text = trim(s.substr(gt + 1, ce - gt - 1));
      p = ce + close.size();
    } else {
      p = gt + 1;
    }
    if (type != "int" && type != "scalar" && type != "model_mat" && type != "dimension" && type != "bool") {
      *msg = "Wrong data type for " + name + "!!!";
      return RW_EFORMAT;
    }
    (*out)[name] = {type, text};
  }
  return RW_OK;
}

int read_project(const std::string& project, HostCase* hc, std::string* msg) {
  std::map<std::string, std::pair<std::string, std::string>> m;
  int rc = read_xml_params(project + ".xml", &m, msg);
  if (rc) return rc;
  bool missing = false;
  std::string miss;
  auto get = [&](const char* name) -> const std::string& {
    static const std::string empty;
    auto it = m.find(name);
    if (it == m.end()) {
      if (!missing) miss = name;
      missing = true;
      return empty;
    }
    return it->second.second;
  };
  auto geti = [&](const char* n) { return std::atoi(get(n).c_str()); };
  auto getd = [&](const char* n) { return std::atof(get(n).c_str()); };
  rw_case_params& p = hc->params;
  std::memset(&p, 0, sizeof(p));
  p.dim = geti("dimension-of-problem");
  p.n_motion = geti("number-of-motion");
  p.periodbound = getd("period-bound") != 0.0;
  if (p.periodbound) {
    const char* names[8] = {"planeleft-A", "planeleft-B", "planeleft-C", "planeleft-D",
                            "planeright-A", "planeright-B", "planeright-C", "planeright-D"};
    for (int k = 0; k < 4; ++k) p.planeleft[k] = getd(names[k]);
    for (int k = 0; k < 4; ++k) p.planeright[k] = getd(names[4 + k]);
  }
  p.np = geti("number-of-particles");
  p.npb = geti("number-of-boundary-particles");
  p.npm = geti("number-of-material-particles");
  p.domain_size[0] = getd("domain-size-x");
  p.domain_size[1] = getd("domain-size-y");
  p.domain_size[2] = getd("domain-size-z");
  p.domain_min[0] = getd("domain-min-x");
  p.domain_min[1] = getd("domain-min-y");
  p.domain_min[2] = getd("domain-min-z");
  p.dr = getd("particle-size");
  p.hdr = getd("h-over-dr");
  p.gravity[0] = getd("acceleration-x");
  p.gravity[1] = getd("acceleration-y");
  p.gravity[2] = getd("acceleration-z");
  p.rho0_m = getd("reference-density-material");
  p.damping = getd("damping");
  p.n_model = geti("number-of-model");
  if (p.n_model < 0 || p.n_model > RW_MODEL_MAX) {
    *msg = "number-of-model out of range";
    return RW_EFORMAT;
  }
  for (int i = 0; i < p.n_model; ++i)
    for (int j = 0; j < RW_MATERIAL_SIZE; ++j) {
      std::string n = "model-" + std::to_string(i) + "-par-" + std::to_string(j);
      p.model_par[i][j] = getd(n.c_str());
    }
  p.stress_shepard_filter = geti("stress-shepard-filter");
  p.dynamic_time_step = geti("dynamic-time-step");
  p.integration_method = geti("integration-method");
  p.viscosity_type = geti("viscosity-type");
  if (p.viscosity_type == 1) p.artificial_viscosity_alpha_m = getd("artificial-viscosity-alpha-material");
  p.cs_m = getd("speed-of-sound-material");
  p.cfl = getd("cfl-number");
  p.artificial_pressure_coefficient_material = getd("artificial-pressure-coefficient-material");
  p.time_max = getd("time-max");
  p.time = getd("time");
  p.dt = getd("time-step");
  p.output_frequency = getd("output-frequency");
  p.output_number = geti("output-number");
  p.output_format = geti("output-format");
  if (missing) {
    *msg = "Error! " + miss + " does not exist in the xml file!";
    return RW_EFORMAT;
  }
  auto wf = m.find("wall-friction-coefficient");
  p.wall_friction = wf == m.end() ? 0.58108 : std::atof(wf->second.second.c_str());
  if (p.np != p.npb + p.npm || p.np <= 0 || p.npb < 0) {
    *msg = "Error! Wrong number of particles ...";
    return RW_EFORMAT;
  }
  if (p.n_motion < 0 || p.n_motion > RW_MOTION_MAX) {
    *msg = "number-of-motion out of range";
    return RW_EFORMAT;
  }
  // .dat (src/loquat_io.cu:222-264): one particle per line, read whole, the lines
  // parsed by several host threads (strtol / strtod, as a line-by-line read would)
  std::FILE* df = std::fopen((project + ".dat").c_str(), "rb");
  if (!df) {
    *msg = "Error! Cannot open " + project + ".dat !";
    return RW_ENOENT;
  }
  std::string buf;
  {
    char chunk[1 << 16];
    size_t got;
    while ((got = std::fread(chunk, 1, sizeof(chunk), df)) > 0) buf.append(chunk, got);
    std::fclose(df);
  }
  const size_t np = (size_t)p.np, npb = (size_t)p.npb;
  hc->codes.assign(4 * np, 0);
  hc->pospres.assign(4 * np, 0.0);
  hc->velrhop.assign(4 * np, 0.0);
  hc->idmassidx.assign(4 * np, 0.0);
  hc->stress.assign(6 * np, 0.0);
  hc->strain.assign(6 * np, 0.0);
  hc->normal.assign(4 * npb, 0.0);
  // the first np lines, each ended by a terminator in place of its newline
  std::vector<size_t> start(np);
  size_t at = 0;
  for (size_t i = 0; i < np; ++i) {
    if (at >= buf.size()) {
      *msg = "Error! " + project + ".dat ends before particle " + std::to_string(i);
      return RW_EFORMAT;
    }
    start[i] = at;
    const size_t nl = buf.find('\n', at);
    if (nl == std::string::npos) {
      at = buf.size();
    } else {
      buf[nl] = '\0';
      at = nl + 1;
    }
  }
  std::vector<size_t> bad_line(io_threads(), np);  // per thread: first malformed line
  auto parse = [&](int t, size_t lo, size_t hi) {
    for (size_t i = lo; i < hi; ++i) {
      const char* c = buf.c_str() + start[i];
      char* e = nullptr;
      bool ok = true;
      auto nextl = [&]() {
        long v = std::strtol(c, &e, 10);
        ok = ok && e != c;
        c = e;
        return (int32_t)v;
      };
      auto nextd = [&]() {
        double v = std::strtod(c, &e);
        ok = ok && e != c;
        c = e;
        return v;
      };
      for (int k = 0; k < 4; ++k) hc->codes[4 * i + k] = nextl();
      for (int k = 0; k < 4; ++k) hc->pospres[4 * i + k] = nextd();
      for (int k = 0; k < 4; ++k) hc->velrhop[4 * i + k] = nextd();
      hc->idmassidx[4 * i + 0] = nextd();
      hc->idmassidx[4 * i + 1] = nextd();
      hc->idmassidx[4 * i + 3] = nextd();
      hc->idmassidx[4 * i + 2] = (double)i;
      for (int k = 0; k < 6; ++k) hc->stress[6 * i + k] = nextd();
      for (int k = 0; k < 6; ++k) hc->strain[6 * i + k] = nextd();
      if (i < npb)
        for (int k = 0; k < 4; ++k) hc->normal[4 * i + k] = nextd();
      if (!ok) {
        bad_line[t] = i;
        return;
      }
    }
  };
  {
    const int nth = np < 8192 ? 1 : (int)bad_line.size();
    std::vector<std::thread> th;
    for (int t = 1; t < nth; ++t) th.emplace_back(parse, t, np * t / nth, np * (t + 1) / nth);
    parse(0, 0, np / nth);
    for (auto& x : th) x.join();
  }
  const size_t bad = *std::min_element(bad_line.begin(), bad_line.end());
  if (bad < np) {
    *msg = "Error! malformed particle line " + std::to_string(bad) + " in " + project + ".dat";
    return RW_EFORMAT;
  }
  // .motion (src/loquat_io.cu:266-311)
  if (p.n_motion > 0) {
    std::ifstream mf(project + ".motion");
    if (!mf) {
      *msg = "Error! Cannot open " + project + ".motion !";
      return RW_ENOENT;
    }
    for (int i = 0; i < p.n_motion; ++i) {
      rw_motion& mo = p.motion[i];
      if (!(mf >> mo.is_translation >> mo.is_rotation)) {
        *msg = "Error! malformed " + project + ".motion";
        return RW_EFORMAT;
      }
      if (mo.is_translation) {
        mf >> mo.n_trans;
        if (mo.n_trans < 0 || mo.n_trans > RW_TABLE_MAX) {
          *msg = "motion table too long";
          return RW_EFORMAT;
        }
        for (int j = 0; j < mo.n_trans; ++j)
          mf >> mo.trans_time[j] >> mo.trans_vel[j][0] >> mo.trans_vel[j][1] >> mo.trans_vel[j][2] >>
              mo.trans_acc[j][0] >> mo.trans_acc[j][1] >> mo.trans_acc[j][2];
      }
      if (mo.is_rotation) {
        mf >> mo.pattern >> mo.pos_rp[0] >> mo.pos_rp[1] >> mo.pos_rp[2] >> mo.rotat_vel[0] >> mo.rotat_vel[1] >>
            mo.rotat_vel[2] >> mo.n_rot;
        if (mo.n_rot < 0 || mo.n_rot > RW_TABLE_MAX) {
          *msg = "motion table too long";
          return RW_EFORMAT;
        }
        for (int j = 0; j < mo.n_rot; ++j)
          mf >> mo.rotat_time[j] >> mo.rotat_acc[j][0] >> mo.rotat_acc[j][1] >> mo.rotat_acc[j][2];
      }
      if (!mf) {
        *msg = "Error! malformed " + project + ".motion";
        return RW_EFORMAT;
      }
    }
  }
  return RW_OK;
}

// Values are printed like the reference's ofstream (default 6 significant digits), here
// and in the particle files.
int write_output_xml(const std::string& path, const rw_case_params& p, int np, int npb, int npm, double time,
                     double dt, int output_number) {
  std::ofstream o(path);
  if (!o) return RW_EIO;
  auto t = [&](const char* n, const char* ty, auto v) { o << "  <" << n << " type=\"" << ty << "\">" << v << "</" << n << ">\n"; };
  o << "<?xml version=\"1.0\" encoding=\"utf-8\" ?>\n<parameters>\n";
  t("dimension-of-problem", "dimension", p.dim);
  t("number-of-motion", "int", p.n_motion);
  t("period-bound", "bool", p.periodbound);
  if (p.periodbound) {
    const char* nm[8] = {"planeleft-A", "planeleft-B", "planeleft-C", "planeleft-D",
                         "planeright-A", "planeright-B", "planeright-C", "planeright-D"};
    for (int k = 0; k < 4; ++k) t(nm[k], "scalar", p.planeleft[k]);
    for (int k = 0; k < 4; ++k) t(nm[4 + k], "scalar", p.planeright[k]);
  }
  t("number-of-particles", "int", np);
  t("number-of-boundary-particles", "int", npb);
  t("number-of-material-particles", "int", npm);
  t("domain-size-x", "scalar", p.domain_size[0]);
  t("domain-size-y", "scalar", p.domain_size[1]);
  t("domain-size-z", "scalar", p.domain_size[2]);
  t("domain-min-x", "scalar", p.domain_min[0]);
  t("domain-min-y", "scalar", p.domain_min[1]);
  t("domain-min-z", "scalar", p.domain_min[2]);
  t("particle-size", "scalar", p.dr);
  t("h-over-dr", "scalar", p.hdr);
  t("acceleration-x", "scalar", p.gravity[0]);
  t("acceleration-y", "scalar", p.gravity[1]);
  t("acceleration-z", "scalar", p.gravity[2]);
  t("reference-density-material", "scalar", p.rho0_m);
  t("damping", "scalar", p.damping);
  t("number-of-model", "int", p.n_model);
  for (int i = 0; i < p.n_model; ++i)
    for (int j = 0; j < RW_MATERIAL_SIZE; ++j) {
      std::string n = "model-" + std::to_string(i) + "-par-" + std::to_string(j);
      t(n.c_str(), "scalar", p.model_par[i][j]);
    }
  t("stress-shepard-filter", "int", p.stress_shepard_filter);
  t("dynamic-time-step", "int", p.dynamic_time_step);
  t("integration-method", "int", p.integration_method);
  t("viscosity-type", "int", p.viscosity_type);
  if (p.viscosity_type == 1) t("artificial-viscosity-alpha-material", "scalar", p.artificial_viscosity_alpha_m);
  t("speed-of-sound-material", "scalar", p.cs_m);
  t("cfl-number", "scalar", p.cfl);
  t("artificial-pressure-coefficient-material", "scalar", p.artificial_pressure_coefficient_material);
  t("time-max", "scalar", p.time_max);
  t("time", "scalar", (float)time);
  t("time-step", "scalar", dt);
  t("output-frequency", "scalar", p.output_frequency);
  t("output-number", "int", output_number);
  t("output-format", "int", p.output_format);
  o << "</parameters>\n";
  return o ? RW_OK : RW_EIO;
}

// Row layout of LoquatIo::SaveParticles format 1 (src/loquat_io.cu:440-461): every live
// particle (boundary and soil) carries four normal columns, deleted particles do not and
// end with a space.  The reference prints normal_m[i] for live soil rows too, reading
// past its npb-entry normal array (src/loquat_io.cu:216,449); those columns are 0 here.
// Rows are formatted by several host threads and written in order.
int write_frame_dat(const std::string& path, const Frame& f) {
  std::FILE* o = std::fopen(path.c_str(), "wb");
  if (!o) return RW_EIO;
  const int live = f.npb + f.npm;
  auto row = [&](size_t q, std::string& s) {
    const int i = (int)q;
    const int32_t* c = &f.codes[4 * i];
    put_i(s, c[0]);
    for (int k = 1; k < 4; ++k) {
      s.push_back(' ');
      put_i(s, c[k]);
    }
    auto g = [&](double v) {
      s.push_back(' ');
      put_g(s, v);
    };
    for (int k = 0; k < 4; ++k) g(f.pos[4 * i + k]);
    for (int k = 0; k < 4; ++k) g(f.vel[4 * i + k]);
    g(f.idm[4 * i + 0]);
    g(f.idm[4 * i + 1]);
    g(f.idm[4 * i + 3]);
    for (int k = 0; k < 6; ++k) g(f.str[6 * i + k]);
    for (int k = 0; k < 6; ++k) g(f.stn[6 * i + k]);
    if (i < f.npb)
      for (int k = 0; k < 4; ++k) g(f.normal[4 * i + k]);
    else if (i < live)
      s.append(" 0 0 0 0");
    else
      s.push_back(' ');
    s.push_back('\n');
  };
  bool ok = put_rows(o, (size_t)f.np, 300, row);
  ok = std::fclose(o) == 0 && ok;
  return ok ? RW_OK : RW_EIO;
}

int write_frame_vtu(const std::string& dir, int output_number, const Frame& f) {
  // Order particles by block id (stable), as the host thrust sort by idmassidx.x does.
  std::vector<int> idx(f.np);
  std::iota(idx.begin(), idx.end(), 0);
  std::stable_sort(idx.begin(), idx.end(), [&](int a, int b) { return (int)f.idm[4 * a] < (int)f.idm[4 * b]; });
  size_t s = 0;
  while (s < idx.size()) {
    const int id = (int)f.idm[4 * idx[s]];
    size_t e = s;
    while (e < idx.size() && (int)f.idm[4 * idx[e]] == id) ++e;
    const size_t n = e - s;
    const std::string path = dir + "/" + std::to_string(id) + "_" + std::to_string(output_number) + ".vtu";
    std::FILE* o = std::fopen(path.c_str(), "wb");
    if (!o) return RW_EIO;
    bool ok = put_text(o, "<?xml version=\"1.0\"?>\n<VTKFile type=\"UnstructuredGrid\" version=\"0.1\" "
                          "byte_order=\"LittleEndian\" compressor=\"vtkZLibDataCompressor\">\n  <UnstructuredGrid "
                          "GhostLevel=\"0\">\n");
    ok = ok && put_text(o, "    <Piece NumberOfPoints=\"" + std::to_string(n) + "\" NumberOfCells=\"" +
                               std::to_string(n) + "\" Name=\"" + std::to_string(id) + "\">\n      <PointData>\n");
    // one DataArray: the block's rows formatted by several threads, each row by fn(i, out)
    auto arr = [&](const char* name, int ncomp, auto fn) {
      std::string h = std::string("        <DataArray type=\"Float64\" Name=\"") + name + "\"";
      if (ncomp > 1) h += " NumberOfComponents=\"" + std::to_string(ncomp) + "\"";
      h += ">\n";
      ok = ok && put_text(o, h);
      ok = ok && put_rows(o, n, 16 * (size_t)ncomp, [&](size_t q, std::string& t) { fn(idx[s + q], t); });
      ok = ok && put_text(o, "</DataArray>\n");
    };
    auto g = [](std::string& t, double v) {
      put_g(t, v);
      t.push_back(' ');
    };
    arr("Material", 1, [&](int i, std::string& t) {
      put_i(t, f.codes[4 * i + 3]);
      t.push_back(' ');
    });
    arr("Ori_ID", 1, [&](int i, std::string& t) { g(t, f.idm[4 * i + 3]); });
    arr("Velocity", 3, [&](int i, std::string& t) {
      for (int k = 0; k < 3; ++k) g(t, f.vel[4 * i + k]);
    });
    arr("Acceleration", 3, [&](int i, std::string& t) {
      for (int k = 0; k < 3; ++k) g(t, f.acc[4 * i + k]);
    });
    arr("Density", 1, [&](int i, std::string& t) { g(t, f.vel[4 * i + 3]); });
    arr("Mass", 1, [&](int i, std::string& t) { g(t, f.idm[4 * i + 1]); });
    if (id < 100)
      arr("Normal", 3, [&](int i, std::string& t) {
        if (i < f.npb)
          for (int k = 0; k < 3; ++k) g(t, f.normal[4 * i + k]);
        else
          t.append("0 0 0 ");
      });
    // six components in the order xx yy zz xy yz xz
    auto six = [&](const std::vector<double>& a, int i, std::string& t) {
      const double* v = &a[6 * (size_t)i];
      for (int k : {0, 1, 2, 3, 5, 4}) g(t, v[k]);
    };
    arr("Stress", 6, [&](int i, std::string& t) { six(f.str, i, t); });
    arr("Strain", 6, [&](int i, std::string& t) { six(f.stn, i, t); });
    ok = ok && put_text(o, "      </PointData>\n      <CellData>\n      </CellData>\n      <Points>\n"
                           "        <DataArray type=\"Float64\" Name=\"Points\" NumberOfComponents=\"3\">\n");
    ok = ok && put_rows(o, n, 48, [&](size_t q, std::string& t) {
      const int i = idx[s + q];
      for (int k = 0; k < 3; ++k) g(t, f.pos[4 * i + k]);
    });
    ok = ok && put_text(o, "</DataArray>\n      </Points>\n      <Cells>\n        <DataArray type=\"Int64\" "
                           "Name=\"connectivity\" format=\"ascii\">\n");
    ok = ok && put_rows(o, n, 8, [&](size_t q, std::string& t) {
      put_i(t, (long long)q);
      t.push_back(' ');
    });
    ok = ok && put_text(o, "</DataArray>\n        <DataArray type=\"Int64\" Name=\"offsets\" format=\"ascii\"> \n");
    ok = ok && put_rows(o, n, 8, [&](size_t q, std::string& t) {
      put_i(t, (long long)q + 1);
      t.push_back(' ');
    });
    ok = ok && put_text(o, "</DataArray>\n        <DataArray type=\"Int64\" Name=\"types\" format=\"ascii\">\n");
    ok = ok && put_rows(o, n, 2, [&](size_t, std::string& t) { t.append("1 "); });
    ok = ok && put_text(o, "</DataArray>\n      </Cells>\n    </Piece>\n  </UnstructuredGrid>\n</VTKFile>\n");
    ok = std::fclose(o) == 0 && ok;
    if (!ok) return RW_EIO;
    s = e;
  }
  return RW_OK;
}

// SaveDatFile layout (src/GenCase.cu:70-116): codes(4) pos(4) velrhop(4) id mass w
// stress(6) strain(6), plus the normal(4) on boundary rows; integers in decimal, reals
// as printf's %.9g (enough digits to give a float back exactly).  Rows are formatted by
// several host threads into separate buffers and written in order.
int write_case_dat(const rw_case* c, const std::string& path) {
  const int np = c->params.np, npb = c->params.npb;
  if (np < 0 || npb < 0 || npb > np) return RW_EINVAL;
  const int nth = (int)std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
  std::vector<std::string> part(nth);
  auto rows = [&](int t) {
    const long lo = (long)np * t / nth, hi = (long)np * (t + 1) / nth;
    std::string& o = part[t];
    o.reserve((size_t)(hi - lo) * 330);
    char buf[64];
    auto put_i = [&](int32_t v) {
      auto r = std::to_chars(buf, buf + sizeof(buf), v);
      o.append(buf, r.ptr);
    };
    auto put_d = [&](double v) {
      o.push_back(' ');
      auto r = std::to_chars(buf, buf + sizeof(buf), v, std::chars_format::general, 9);
      o.append(buf, r.ptr);
    };
    for (long i = lo; i < hi; ++i) {
      const int32_t* cc = c->codes + 4 * i;
      put_i(cc[0]);
      for (int k = 1; k < 4; ++k) {
        o.push_back(' ');
        put_i(cc[k]);
      }
      for (int k = 0; k < 4; ++k) put_d(c->pospres[4 * i + k]);
      for (int k = 0; k < 4; ++k) put_d(c->velrhop[4 * i + k]);
      put_d(c->idmassidx[4 * i + 0]);
      put_d(c->idmassidx[4 * i + 1]);
      put_d(c->idmassidx[4 * i + 3]);
      for (int k = 0; k < 6; ++k) put_d(c->stress[6 * i + k]);
      for (int k = 0; k < 6; ++k) put_d(c->strain[6 * i + k]);
      if (i < npb)
        for (int k = 0; k < 4; ++k) put_d(c->normal[4 * i + k]);
      o.push_back('\n');
    }
  };
  std::vector<std::thread> th;
  for (int t = 1; t < nth; ++t) th.emplace_back(rows, t);
  rows(0);
  for (auto& x : th) x.join();
  std::FILE* f = std::fopen(path.c_str(), "wb");
  if (!f) return RW_EIO;
  bool ok = true;
  for (auto& s : part) ok = ok && std::fwrite(s.data(), 1, s.size(), f) == s.size();
  ok = std::fclose(f) == 0 && ok;
  return ok ? RW_OK : RW_EIO;
}

}  // namespace rw

extern "C" rw_status rw_write_case_dat(const rw_case* c, const char* path) {
  if (!c || !path) return RW_EINVAL;
  try {
    return rw::write_case_dat(c, path);
  } catch (...) {
    return RW_ENOMEM;
  }
}
