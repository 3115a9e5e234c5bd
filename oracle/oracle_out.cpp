// The reference's binary output writers and its calendar, restated for the CPU oracle — TEST
// INFRASTRUCTURE ONLY (see oracle.hpp).
//
// outp (si3d_utils.f90:2484-2602, the ptrack file "si3d_3D"), outz (:2373-2481, "tracer_<n>") and
// outh (:2142-2334, "plane_<k>") write Fortran unformatted sequential files: every WRITE is one
// record framed by its byte length as a 4-byte little-endian integer before and after.  Integers are
// 4 bytes and REAL values are written as 4-byte IEEE floats (the default-REAL build that the
// downstream readers expect), each state value rounded to the nearest float.
#include <cmath>
#include <cstring>

#include "oracle.hpp"

namespace orc {

// compute_date (si3d_utils.f90:3546-3674).  REAL as double; NINT rounds half away from zero; the
// month table keeps its changes between calls (an initialised local variable is SAVEd).
void compute_date(Model& m, double itime_sec) {
  Date& D = m.date;
  const Inp& p = m.in;
  auto leap = [](int y) { return y % 4 == 0; };
  if (itime_sec == 0) {
    D.iyrp = p.iyr0; D.imonp = p.imon0; D.idayp = p.iday0; D.ihrp = p.ihr0; D.isecp = D.isec0;
    D.iyr = p.iyr0; D.imon = p.imon0; D.iday = p.iday0; D.ihr = p.ihr0; D.isec = D.isec0;
    if (leap(D.iyrp)) D.month[1] = 29;
    return;
  }
  D.isecp = D.isecp + itime_sec;
  if (D.isecp < 86400) {
    D.isec = D.isecp;
    const double hrs = D.isec / 3600.;
    D.ihrp = (int)std::lround(hrs * 100.);
    D.ihr = D.ihrp;
    return;
  }
  D.idayp = (int)(D.idayp + D.isecp / 86400);
  D.isecp = std::fmod(D.isecp, 86400.);
  D.isec = D.isecp;
  const double hrs = D.isec / 3600.;
  D.ihrp = (int)std::lround(hrs * 100.);
  D.ihr = D.ihrp;
  if (D.imonp == 2) {
    D.month[1] = 28;
    if (leap(D.iyrp)) D.month[1] = 29;
  }
  if (D.idayp <= D.month[D.imonp - 1]) {
    D.iday = D.idayp;
    return;
  }
  const int max_possible_months = (int)(itime_sec / 2500000 + 1);
  for (int j = 1; j <= max_possible_months; ++j) {
    D.idayp = D.idayp - D.month[D.imonp - 1];
    D.imonp = D.imonp + 1;
    if (D.imonp == 13) {
      D.imonp = 1;
      D.iyrp = D.iyrp + 1;
      D.month[1] = leap(D.iyrp) ? 29 : 28;
    }
    if (D.idayp <= D.month[D.imonp - 1]) {
      D.iday = D.idayp;
      break;
    }
  }
  D.imon = D.imonp;
  D.iyr = D.iyrp;
}

namespace {

struct Record {
  std::vector<char> b;
  void i4(int32_t v) { put(&v, 4); }
  void f4(double v) { const float f = (float)v; put(&f, 4); }
  void put(const void* q, size_t n) { const char* c = static_cast<const char*>(q); b.insert(b.end(), c, c + n); }
};

bool emit(Model& m, const std::shared_ptr<FILE>& f, const Record& r) {
  const int32_t len = (int32_t)r.b.size();
  bool ok = std::fwrite(&len, 4, 1, f.get()) == 1 && std::fwrite(r.b.data(), 1, r.b.size(), f.get()) == r.b.size() &&
            std::fwrite(&len, 4, 1, f.get()) == 1;
  std::fflush(f.get());
  if (!ok) m.err = "output: write failed";
  return ok;
}

std::shared_ptr<FILE> open_out(Model& m, const std::string& name) {
  FILE* f = std::fopen((m.dir + "/" + name).c_str(), "wb");
  if (!f) { m.err = "output: cannot open " + name; return nullptr; }
  return std::shared_ptr<FILE>(f, [](FILE* q) { std::fclose(q); });
}

void stamp(const Model& m, Record& r, int n) {
  r.i4(n); r.i4(m.date.iyr); r.i4(m.date.imon); r.i4(m.date.iday); r.f4((double)(float)m.date.ihr);
}

int points3(const Model& m) {
  int n = 0;
  for (int l = 1; l <= m.lm; ++l) n += m.kmz(l) + 1 - m.k1 + 1;
  return n;
}

// outp (si3d_utils.f90:2484-2602)
bool outp(Model& m, int n) {
  Record r;
  if (n == 0) {
    const int apxml = std::abs(m.in.ipxml);
    m.f_ptrack = open_out(m, "si3d_3D");
    if (!m.f_ptrack) return false;
    Record a, b;
    a.i4((m.nts - m.in.itspf) / std::max(apxml, 1));
    b.i4(points3(m));
    if (!emit(m, m.f_ptrack, a) || !emit(m, m.f_ptrack, b)) return false;
  }
  stamp(m, r, n);
  for (int l = 1; l <= m.lm; ++l)
    for (int k = m.k1; k <= m.kmz(l) + 1; ++k) {
      if (n == 0) { r.f4(m.l2i(l)); r.f4(m.l2j(l)); r.f4(k); }
      r.f4(m.hp(k, l)); r.f4(m.up(k, l)); r.f4(m.vp(k, l)); r.f4(m.wp(k, l)); r.f4(m.salp(k, l));
    }
  return emit(m, m.f_ptrack, r);
}

// outz (si3d_utils.f90:2373-2481)
bool outz(Model& m, int n) {
  if (m.in.ntr <= 0) return true;
  if (n == 0) {
    m.f_tracer.clear();
    for (int j = 1; j <= m.in.ntr; ++j) {
      auto f = open_out(m, "tracer_" + std::to_string(j));
      if (!f) return false;
      Record a, b;
      a.i4((m.nts - m.in.itspftr) / std::max(m.in.iotr, 1));
      b.i4(points3(m));
      if (!emit(m, f, a) || !emit(m, f, b)) return false;
      m.f_tracer.push_back(f);
    }
  }
  for (int t = 1; t <= m.in.ntr; ++t) {
    const F3& c = m.tracer[t - 1];
    Record r;
    stamp(m, r, n);
    for (int l = 1; l <= m.lm; ++l)
      for (int k = m.k1; k <= m.kmz(l) + 1; ++k) {
        if (n == 0) { r.f4(m.l2i(l)); r.f4(m.l2j(l)); r.f4(k); }
        r.f4(c(k, l));
      }
    if (!emit(m, m.f_tracer[t - 1], r)) return false;
  }
  return true;
}

// outh (si3d_utils.f90:2142-2334) with CountPlaneCells (:2337-2368): one file per plane; a plane
// below the deepest layer (kp > km) holds every column's bottom layer.
bool outh(Model& m, int n) {
  const real ZERO = 0.0;
  if (n == 0) {
    m.f_plane.clear();
    for (int kp : m.in.p_out) {
      if (kp < m.k1) { m.err = "ERROR: Output plane is not in DOMAIN"; return false; }
      auto f = open_out(m, "plane_" + std::to_string(kp));
      if (!f) return false;
      int cnt = 0;
      for (int l = 1; l <= m.lm; ++l)
        if (m.km < kp || m.kmz(l) >= kp) ++cnt;
      Record a, b;
      a.i4((m.nts - m.in.itspfh) / std::max(m.in.iop, 1));
      b.i4(cnt);
      if (!emit(m, f, a) || !emit(m, f, b)) return false;
      m.f_plane.push_back(f);
    }
  }
  for (size_t j = 0; j < m.in.p_out.size(); ++j) {
    const int kp = m.in.p_out[j];
    Record r;
    stamp(m, r, n);
    for (int l = 1; l <= m.lm; ++l) {
      int kb;
      if (kp > m.km) kb = m.kmz(l);
      else if (m.kmz(l) < kp) continue;
      else kb = kp;
      const double sal = (m.hp(kb, l) <= ZERO) ? -99. : m.salp(kb, l);
      if (n == 0) {
        r.f4(m.l2i(l)); r.f4(m.l2j(l));
        r.f4(m.up(kb, l)); r.f4(m.vp(kb, l)); r.f4(m.wp(kb, l));
      } else {
        r.f4((m.up(kb, l) + m.up(kb, m.lWC(l))) / 2.);
        r.f4((m.vp(kb, l) + m.vp(kb, m.lSC(l))) / 2.);
        r.f4((m.wp(kb, l) + m.wp(kb + 1, l)) / 2.);
      }
      r.f4(sal);
      r.f4(0.5 * (m.Av(kb, l) + m.Av(kb + 1, l)));
      r.f4(m.s(l));
    }
    if (!emit(m, m.f_plane[j], r)) return false;
  }
  return true;
}

}  // namespace

// The output calls of the time loop (si3d.f90:430-438; the initial ones :89-100 with n = 0).
// outs (si3d_utils.f90:2605-2760), ipxml < 0: the Gr viewer's XML header on the first call, the two
// binary space files opened (and left empty: outs_bin, :2763, has no caller).  runNumber, the
// wall-clock date_and_time, is written as 12 zeros here; a comparison skips that line.
static bool outs(Model& m) {
  if (m.space_written) return true;
  const Inp& p = m.in;
  FILE* f = std::fopen((m.dir + "/spacefile.xml").c_str(), "w");
  if (!f) { m.err = "Error opening spacefile.xml"; return false; }
  for (const char* b : {"/spacefile2d.bin", "/spacefile3d.bin"}) {
    FILE* g = std::fopen((m.dir + b).c_str(), "wb");
    if (!g) { std::fclose(f); m.err = "Error opening space file"; return false; }
    std::fclose(g);
  }
  auto ch = [](long v) { return std::string("\"") + std::to_string(v) + "\""; };   // int_to_char(v, 0)
  const int im = m.im, jm = m.jm;
  std::fprintf(f, "<?xml version=\"1.0\"?>\n");
  std::fprintf(f, " \n");
  std::fprintf(f, "<!-- Si3D Output for Gr -->\n");
  std::fprintf(f, "<!-- xml header file for binary spacefiles -->\n");
  // FORMAT 1 (:2651-2655)
  std::fprintf(f, "<!-- Run Parameters:  dt =%5.2f s  dz =%5.2f m  im =%5d  jm =%5d\n", p.idt, m.ddz, im, jm);
  std::fprintf(f, "     itrsca =%2d  itrap =%2d  cd = %7.4f  ismooth =%2d  beta =%6.3f  niter =%2d\n", p.itrsca,
               p.itrap, p.cd, p.ismooth, p.beta, p.niter);
  std::fprintf(f, "     itrmom =%2d  f =%7.4f  wa =%8.1f -->\n", p.itrmom, p.f, p.wa);
  std::fprintf(f, " \n");
  std::fprintf(f, "<gov.usgs.gr>\n");
  std::fprintf(f, "   <obj class=\"gov.usgs.sfhydro.si3d.Si3dOutput\"\n");
  std::string title = p.title;
  while (!title.empty() && title.back() == ' ') title.pop_back();
  std::fprintf(f, "        runTitle=\"%s\"\n", title.c_str());
  std::fprintf(f, "        runNumber=\"000000000000\"\n");
  const long idt2 = (long)p.ipxml * (long)p.idt;
  const Date keep = m.date;
  if (p.itspf == 0) {
    compute_date(m, 0.0);
  } else {
    long itspf1 = (p.itspf / idt2) * idt2;
    if (p.itspf % idt2 != 0) itspf1 = itspf1 + idt2;
    compute_date(m, (double)itspf1);
  }
  const int ihr2 = (int)(m.date.isec / 3600);
  int isec2 = (int)(m.date.isec - ihr2 * 3600);
  const int imin2 = isec2 / 60;
  isec2 = isec2 - imin2 * 60;
  std::fprintf(f, "        startTime=\"%4d/%02d/%02d %02d:%02d:%02d\" timeStepInSeconds=%s>\n", m.date.iyr, m.date.imon,
               m.date.iday, ihr2, imin2, isec2, ch(idt2).c_str());
  m.date = keep;   // compute_date(0.0) returns the calendar to the start of the run
  std::fprintf(f, " \n");
  const char* blocks[2][3] = {{"2-D x-y Variables", "spacefile2d.bin", "2-D Variables"},
                              {"3-D Variables", "spacefile3d.bin", "3-D Variables"}};
  for (int b = 0; b < 2; ++b) {
    std::fprintf(f, "      <obj class=\"gov.usgs.gr.GrObjectContainer\" title=\"%s\">\n", blocks[b][0]);
    std::fprintf(f, "         <dataseries class=\"gov.usgs.gr.data.RafDataSeries\"\n");
    std::fprintf(f, "            file=\"%s\"\n", blocks[b][1]);
    std::fprintf(f, "            title=\"%s\" numDimensions=%s>\n", blocks[b][2], ch(b == 0 ? 1 : 4).c_str());
    if (b == 0) {
      std::fprintf(f, "            <dim num=\"0\" title=\"Zeta\" units=\"meters\" unitScale=\"0.0001\"/>\n");
    } else {
      std::fprintf(f, "            <dim num=\"0\" title=\"u\" units=\"m/s\" unitScale=\"0.0001\"/>\n");
      std::fprintf(f, "            <dim num=\"1\" title=\"v\" units=\"m/s\" unitScale=\"0.0001\"/>\n");
      std::fprintf(f, "            <dim num=\"2\" title=\"w\" units=\"m/s\" unitScale=\"0.00001\"/>\n");
      std::fprintf(f, "            <dim num=\"3\" title=\"dz\" units=\"m**2/s\" unitScale=\"0.0001\"/>\n");
    }
    std::fprintf(f, " \n");
    std::fprintf(f, "         </dataseries>\n");
    std::fprintf(f, "      </obj>\n");
    if (b == 0) std::fprintf(f, " \n");
  }
  std::fprintf(f, "   </obj>\n");
  std::fprintf(f, "</gov.usgs.gr>\n");
  std::fprintf(f, " \n");
  std::fclose(f);
  m.space_written = true;
  return true;
}

bool write_outputs(Model& m, int n) {
  const Inp& p = m.in;
  const int apxml = std::abs(p.ipxml);
  if (p.ipxml < 0 && !outs(m)) return false;   // called at n = 0 and every step; writes once
  if (p.iop > 0 && (n == 0 || (n >= p.itspfh && n % std::max(p.iop, 1) == 0)) && !outh(m, n)) return false;
  if (p.iotr > 0 && (n == 0 || n % std::max(p.iotr, 1) == 0) && !outz(m, n)) return false;
  if (p.ipxml > 0 && (n == 0 || (n >= p.itspf && n % std::max(apxml, 1) == 0)) && !outp(m, n)) return false;
  return true;
}

}  // namespace orc
