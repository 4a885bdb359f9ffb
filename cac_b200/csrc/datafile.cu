// Data files in the reference's read_data format: the sections the force path
// uses (header counts and box, Masses, Element Types, Atoms, Velocities,
// Elements, Nodes, Node Velocities) for one atom type and one element type
// (Hex, one atom per cell, 9x9x9 lattice sites, 2x2x2 integration points),
// read straight into host arrays or a context, and written back from one.
//
// Reference: ReadData::command and its section readers (read_data.cpp:339-367
// and the AtomVec/ElementVec data parsers, element_vec_cac.cpp:300-470);
// write_data / ElementVec write routines (element_vec_cac.cpp:1177-1300).
// Lines are "tag type x y z" (Atoms), "tag vx vy vz" (Velocities),
// "tag etype xc yc zc" (Elements), "etag node basis type x y z" (Nodes) and
// "etag node basis vx vy vz" (Node Velocities); tags run from 1.
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/cacb200.h"

namespace {

thread_local std::string data_error;

struct DataFile {
  int na = 0, ne = 0;
  double lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
  double mass = 0.0;
  std::vector<double> x, v, nodex, nodev;
};

int fail(const std::string &msg) {
  data_error = msg;
  return CACB200_EINVAL;
}

std::string trim(const std::string &s) {
  size_t a = s.find_first_not_of(" \t\r"), b = s.find_last_not_of(" \t\r");
  if (a == std::string::npos) return "";
  std::string t = s.substr(a, b - a + 1);
  size_t h = t.find('#');
  if (h != std::string::npos) t = trim(t.substr(0, h));
  return t;
}

// Parses the file; with counts_only the sections are skipped.
int parse(const char *path, DataFile &d, bool counts_only) {
  if (!path) return fail("no path");
  std::ifstream in(path);
  if (!in) return fail(std::string("cannot open ") + path);
  std::string line;
  std::getline(in, line);   // title
  int atom_types = 1, elem_types = 0;
  bool have_box[3] = {false, false, false};
  std::string section;
  // header
  while (std::getline(in, line)) {
    std::string t = trim(line);
    if (t.empty()) continue;
    std::istringstream ss(t);
    if (t.find("xlo xhi") != std::string::npos) {
      ss >> d.lo[0] >> d.hi[0];
      have_box[0] = true;
    } else if (t.find("ylo yhi") != std::string::npos) {
      ss >> d.lo[1] >> d.hi[1];
      have_box[1] = true;
    } else if (t.find("zlo zhi") != std::string::npos) {
      ss >> d.lo[2] >> d.hi[2];
      have_box[2] = true;
    } else if (t.find("xy xz yz") != std::string::npos) {
      return fail("triclinic boxes are not supported");
    } else if (t.find("element types") != std::string::npos) {
      ss >> elem_types;
    } else if (t.find("atom types") != std::string::npos) {
      ss >> atom_types;
    } else if (t.find("elements") != std::string::npos) {
      ss >> d.ne;
    } else if (t.find("atoms") != std::string::npos) {
      ss >> d.na;
    } else if (std::isalpha((unsigned char)t[0])) {
      section = t;
      break;
    }
  }
  if (!(have_box[0] && have_box[1] && have_box[2])) return fail("box bounds missing");
  if (d.na < 0 || d.ne < 0) return fail("negative counts");
  if (atom_types != 1) return fail("exactly one atom type is supported");
  if (d.ne && elem_types != 1) return fail("exactly one element type is supported");
  // with counts_only the data sections are skipped (Masses and Element Types
  // are still read, wherever they are)
  std::vector<char> got_x, got_n;
  if (!counts_only) {
    d.x.assign(3 * (size_t)d.na, 0.0);
    d.v.assign(3 * (size_t)d.na, 0.0);
    d.nodex.assign(24 * (size_t)d.ne, 0.0);
    d.nodev.assign(24 * (size_t)d.ne, 0.0);
    got_x.assign(d.na, 0);
    got_n.assign(8 * (size_t)d.ne, 0);
  }
  bool have_mass = false;
  while (!section.empty()) {
    std::string next;
    const bool skip = counts_only && section != "Masses" && section != "Element Types";
    while (std::getline(in, line)) {
      std::string t = trim(line);
      if (t.empty()) continue;
      if (std::isalpha((unsigned char)t[0])) {
        next = t;
        break;
      }
      if (skip) continue;
      const char *p = t.c_str();
      char *q;
      if (section == "Masses") {
        long ty = std::strtol(p, &q, 10);
        double m = std::strtod(q, &q);
        if (ty == 1) {
          d.mass = m;
          have_mass = true;
        }
      } else if (section == "Element Types") {
        // "id Hex apc ncx ncy ncz ngx ngy ngz"
        std::istringstream ss(t);
        int id, apc, n1, n2, n3, g1, g2, g3;
        std::string style;
        ss >> id >> style >> apc >> n1 >> n2 >> n3 >> g1 >> g2 >> g3;
        if (!ss || style != "Hex" || apc != 1 || n1 != 9 || n2 != 9 || n3 != 9 || g1 != 2 || g2 != 2 ||
            g3 != 2)
          return fail("element type must be Hex, 1 atom per cell, 9x9x9 sites, 2x2x2 Gauss points");
      } else if (section == "Atoms") {
        long tag = std::strtol(p, &q, 10);
        long ty = std::strtol(q, &q, 10);
        if (tag < 1 || tag > d.na) return fail("atom tag out of range");
        if (ty != 1) return fail("atom type out of range");
        for (int k = 0; k < 3; k++) d.x[3 * (tag - 1) + k] = std::strtod(q, &q);
        got_x[tag - 1] = 1;
      } else if (section == "Velocities") {
        long tag = std::strtol(p, &q, 10);
        if (tag < 1 || tag > d.na) return fail("velocity tag out of range");
        for (int k = 0; k < 3; k++) d.v[3 * (tag - 1) + k] = std::strtod(q, &q);
      } else if (section == "Elements") {
        long tag = std::strtol(p, &q, 10);
        if (tag < 1 || tag > d.ne) return fail("element tag out of range");
      } else if (section == "Nodes" || section == "Node Velocities") {
        long et = std::strtol(p, &q, 10);
        long nd = std::strtol(q, &q, 10);
        long basis = std::strtol(q, &q, 10);
        if (et < 1 || et > d.ne || nd < 1 || nd > 8 || basis != 1) return fail("node index out of range");
        double *dst;
        if (section == "Nodes") {
          std::strtol(q, &q, 10);   // atom type of the node
          dst = &d.nodex[24 * (et - 1) + 3 * (nd - 1)];
          got_n[8 * (et - 1) + (nd - 1)] = 1;
        } else {
          dst = &d.nodev[24 * (et - 1) + 3 * (nd - 1)];
        }
        for (int k = 0; k < 3; k++) dst[k] = std::strtod(q, &q);
      } else {
        return fail("unsupported section: " + section);
      }
    }
    section = next;
  }
  if (!have_mass) return fail("mass of atom type 1 missing");
  if (!counts_only) {
    for (char g : got_x)
      if (!g) return fail("an atom has no line in Atoms");
    for (char g : got_n)
      if (!g) return fail("a node has no line in Nodes");
  }
  return CACB200_OK;
}

std::string fmt(double v) {
  char b[40];
  std::snprintf(b, sizeof(b), "%.17g", v);
  return b;
}

int write(const char *path, int na, int ne, const double lo[3], const double hi[3], double mass, const double *x,
          const double *v, const double *nodex, const double *nodev) {
  if (!path) return fail("no path");
  std::FILE *f = std::fopen(path, "w");
  if (!f) return fail(std::string("cannot write ") + path);
  std::fprintf(f, "CAC data file written by cac_b200\n\n%d atoms\n%d elements\n1 atom types\n1 element types\n\n", na,
               ne);
  const char *ax[3] = {"x", "y", "z"};
  for (int d = 0; d < 3; d++)
    std::fprintf(f, "%s %s %slo %shi\n", fmt(lo[d]).c_str(), fmt(hi[d]).c_str(), ax[d], ax[d]);
  std::fprintf(f, "\nMasses\n\n1 %s\n\nElement Types\n\n1 Hex 1 9 9 9 2 2 2\n\n", fmt(mass).c_str());
  if (na) {
    std::fprintf(f, "Atoms\n\n");
    for (int i = 0; i < na; i++)
      std::fprintf(f, "%d 1 %s %s %s\n", i + 1, fmt(x[3 * i]).c_str(), fmt(x[3 * i + 1]).c_str(),
                   fmt(x[3 * i + 2]).c_str());
    std::fprintf(f, "\nVelocities\n\n");
    for (int i = 0; i < na; i++)
      std::fprintf(f, "%d %s %s %s\n", i + 1, fmt(v[3 * i]).c_str(), fmt(v[3 * i + 1]).c_str(),
                   fmt(v[3 * i + 2]).c_str());
    std::fprintf(f, "\n");
  }
  if (ne) {
    std::fprintf(f, "Elements\n\n");
    for (int e = 0; e < ne; e++) {
      double c[3] = {0, 0, 0};
      for (int k = 0; k < 8; k++)
        for (int d = 0; d < 3; d++) c[d] += nodex[24 * e + 3 * k + d];
      std::fprintf(f, "%d 1 %s %s %s\n", e + 1, fmt(c[0] / 8).c_str(), fmt(c[1] / 8).c_str(), fmt(c[2] / 8).c_str());
    }
    std::fprintf(f, "\nNodes\n\n");
    for (int e = 0; e < ne; e++)
      for (int k = 0; k < 8; k++) {
        const double *p = nodex + 24 * e + 3 * k;
        std::fprintf(f, "%d %d 1 1 %s %s %s\n", e + 1, k + 1, fmt(p[0]).c_str(), fmt(p[1]).c_str(),
                     fmt(p[2]).c_str());
      }
    std::fprintf(f, "\nNode Velocities\n\n");
    for (int e = 0; e < ne; e++)
      for (int k = 0; k < 8; k++) {
        const double *p = nodev + 24 * e + 3 * k;
        std::fprintf(f, "%d %d 1 %s %s %s\n", e + 1, k + 1, fmt(p[0]).c_str(), fmt(p[1]).c_str(),
                     fmt(p[2]).c_str());
      }
    std::fprintf(f, "\n");
  }
  bool ok = std::ferror(f) == 0;
  ok = (std::fclose(f) == 0) && ok;
  return ok ? CACB200_OK : fail(std::string("write failed: ") + path);
}

}  // namespace

extern "C" {

const char *cacb200_data_last_error(void) { return data_error.c_str(); }

int cacb200_data_counts(const char *path, int *natoms, int *nelements, double boxlo[3], double boxhi[3],
                        double *mass) {
  DataFile d;
  int rc = parse(path, d, true);
  if (rc) return rc;
  if (natoms) *natoms = d.na;
  if (nelements) *nelements = d.ne;
  for (int k = 0; k < 3; k++) {
    if (boxlo) boxlo[k] = d.lo[k];
    if (boxhi) boxhi[k] = d.hi[k];
  }
  if (mass) *mass = d.mass;
  return CACB200_OK;
}

int cacb200_data_read(const char *path, double *x, double *v, double *nodex, double *nodev) {
  DataFile d;
  int rc = parse(path, d, false);
  if (rc) return rc;
  if (d.na && (!x || !v)) return fail("null atom arrays");
  if (d.ne && (!nodex || !nodev)) return fail("null node arrays");
  if (d.na) {
    std::memcpy(x, d.x.data(), sizeof(double) * d.x.size());
    std::memcpy(v, d.v.data(), sizeof(double) * d.v.size());
  }
  if (d.ne) {
    std::memcpy(nodex, d.nodex.data(), sizeof(double) * d.nodex.size());
    std::memcpy(nodev, d.nodev.data(), sizeof(double) * d.nodev.size());
  }
  return CACB200_OK;
}

int cacb200_data_write(const char *path, int natoms, int nelements, const double boxlo[3], const double boxhi[3],
                       double mass, const double *x, const double *v, const double *nodex, const double *nodev) {
  if (natoms < 0 || nelements < 0 || !boxlo || !boxhi || (natoms && (!x || !v)) ||
      (nelements && (!nodex || !nodev)))
    return fail("invalid arguments");
  return write(path, natoms, nelements, boxlo, boxhi, mass, x, v, nodex, nodev);
}

int cacb200_read_data(cacb200_ctx *ctx, const char *path) {
  if (!ctx) return CACB200_EINVAL;
  DataFile d;
  int rc = parse(path, d, false);
  if (rc) return rc;
  if (d.na == 0) d.x.resize(3), d.v.resize(3);
  if (d.ne == 0) d.nodex.resize(24), d.nodev.resize(24);
  return cacb200_upload_system(ctx, d.lo, d.hi, d.na, d.x.data(), d.v.data(), d.ne, d.nodex.data(), d.nodev.data(),
                               d.mass);
}

int cacb200_write_data(cacb200_ctx *ctx, const char *path) {
  if (!ctx) return CACB200_EINVAL;
  int na = 0, ne = 0;
  int rc = cacb200_counts(ctx, &na, &ne, nullptr);
  if (rc) return rc;
  double lo[3], hi[3], mass;
  rc = cacb200_get_box(ctx, lo, hi, &mass);
  if (rc) return rc;
  std::vector<double> x(3 * (size_t)std::max(na, 1)), v(x.size()), nx(24 * (size_t)std::max(ne, 1)), nv(nx.size());
  rc = cacb200_get_state(ctx, x.data(), v.data(), nx.data(), nv.data());
  if (rc) return rc;
  return write(path, na, ne, lo, hi, mass, x.data(), v.data(), nx.data(), nv.data());
}

}  // extern "C"
