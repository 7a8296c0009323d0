// .stinput reader and .rays writer: the SolTrace CLI's file front end, as library calls.
//
// The .stinput text format is the one the reference's strace reader consumes
// (coretrace/strace/main.cpp:78-397): a "# SOLTRACE VERSION x.y.z INPUT FILE" line, the
// sun (shape, position or latitude/day/hour, optional user sunshape table), the optical
// property pairs (one line per face, optional angle tables), and the stages with their
// elements (one tab-separated line of 29 fields per element).  The .rays text format is
// the one strace writes (main.cpp:399-483): the sun box and ray counts, then one line per
// intersection record in the reference's readback order.
//
// Only stapi.h calls are made here, so the same source serves any library exporting
// that API.  Errors go to the context's messages through st_input_report(), which the
// library linking this file provides.
#include <cctype>
#include <cerrno>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "stapi.h"
#include "st_b200.h"

extern "C" void st_input_report(st_context_t ctx, const char *msg);

namespace {

struct Reader {
    FILE *fp = nullptr;
    st_context_t ctx = nullptr;
    int line_no = 0;
    std::string line;

    // next line without its end-of-line characters; false at end of file
    bool next() {
        line.clear();
        int c;
        bool any = false;
        while ((c = fgetc(fp)) != EOF) {
            any = true;
            if (c == '\n') break;
            line.push_back(char(c));
        }
        if (!any) return false;
        if (!line.empty() && line.back() == '\r') line.pop_back();
        ++line_no;
        return true;
    }

    bool fail(const std::string &what) {
        char buf[64];
        snprintf(buf, sizeof buf, "line %d: ", line_no);
        st_input_report(ctx, (std::string(".stinput ") + buf + what).c_str());
        return false;
    }
};

// fields separated by single tabs, empty fields kept (an empty surface-file column)
std::vector<std::string> tab_fields(const std::string &s) {
    std::vector<std::string> out;
    size_t a = 0;
    for (;;) {
        const size_t b = s.find('\t', a);
        if (b == std::string::npos) {
            out.push_back(s.substr(a));
            return out;
        }
        out.push_back(s.substr(a, b - a));
        a = b + 1;
    }
}

// whitespace-separated words
std::vector<std::string> words(const std::string &s) {
    std::vector<std::string> out;
    size_t i = 0;
    while (i < s.size()) {
        while (i < s.size() && isspace((unsigned char)s[i])) ++i;
        size_t j = i;
        while (j < s.size() && !isspace((unsigned char)s[j])) ++j;
        if (j > i) out.push_back(s.substr(i, j - i));
        i = j;
    }
    return out;
}

bool num(const std::string &s, double &v) {
    const char *p = s.c_str();
    char *end = nullptr;
    errno = 0;
    v = strtod(p, &end);
    return end != p;
}

double num_or0(const std::string &s) {
    double v = 0.0;
    return num(s, v) ? v : 0.0;
}

// "KEY v KEY v ..." lines: the value following keyword `key`
bool keyed(const std::vector<std::string> &w, const char *key, double &v) {
    for (size_t i = 0; i + 1 < w.size(); ++i)
        if (w[i] == key) return num(w[i + 1], v);
    return false;
}

// a count after a fixed prefix ("OPTICS LIST COUNT\t3")
bool count_after(const std::string &line, const char *prefix, int &n) {
    const size_t k = strlen(prefix);
    if (line.compare(0, k, prefix) != 0) return false;
    double v = 0;
    if (!num(line.substr(k), v) || v < 0) return false;
    n = int(v);
    return true;
}

bool two_numbers(const std::string &line, double &a, double &b) {
    const auto w = words(line);
    return w.size() >= 2 && num(w[0], a) && num(w[1], b);
}

bool read_sun(Reader &r) {
    if (!r.next()) return r.fail("missing SUN line");
    auto w = words(r.line);
    if (w.empty() || w[0] != "SUN") return r.fail("expected SUN");
    double ps = 0, sigma = 0, half = 0;
    char shape = 'g';
    keyed(w, "PTSRC", ps);
    for (size_t i = 0; i + 1 < w.size(); ++i)
        if (w[i] == "SHAPE") shape = char(tolower((unsigned char)w[i + 1][0]));
    keyed(w, "SIGMA", sigma);
    keyed(w, "HALFWIDTH", half);
    if (st_sun(r.ctx, ps != 0 ? 1 : 0, shape, shape == 'g' ? sigma : half) < 0) return r.fail("st_sun failed");

    if (!r.next()) return r.fail("missing XYZ line");
    w = words(r.line);
    if (w.size() < 4 || w[0] != "XYZ") return r.fail("expected XYZ");
    double x = 0, y = 0, z = 0, use_ldh = 0, lat = 0, day = 0, hour = 0;
    num(w[1], x);
    num(w[2], y);
    num(w[3], z);
    keyed(w, "USELDH", use_ldh);
    for (size_t i = 0; i + 3 < w.size(); ++i)
        if (w[i] == "LDH") {
            num(w[i + 1], lat);
            num(w[i + 2], day);
            num(w[i + 3], hour);
        }
    if (use_ldh != 0) st_sun_position(r.ctx, lat, day, hour, &x, &y, &z);
    st_sun_xyz(r.ctx, x, y, z);

    if (!r.next()) return r.fail("missing USER SHAPE DATA line");
    int n = 0;
    if (!count_after(r.line, "USER SHAPE DATA", n)) return r.fail("expected USER SHAPE DATA");
    if (n > 0) {
        std::vector<double> ang(n), inten(n);
        for (int i = 0; i < n; ++i) {
            if (!r.next() || !two_numbers(r.line, ang[i], inten[i])) return r.fail("bad sunshape table row");
        }
        // as the CLI does (strace/main.cpp:114-129), the setter's result is not checked: a table of
        // two rows or fewer is refused by st_sun_userdata and leaves the sunshape table unset
        st_sun_userdata(r.ctx, st_uint_t(n), ang.data(), inten.data());
    }
    return true;
}

bool read_table(Reader &r, int n, std::vector<double> &a, std::vector<double> &v) {
    a.assign(size_t(n), 0.0);
    v.assign(size_t(n), 0.0);
    for (int i = 0; i < n; ++i)
        if (!r.next() || !two_numbers(r.line, a[i], v[i])) return r.fail("bad property table row");
    return true;
}

bool read_face(Reader &r, int iopt, int fb) {
    if (!r.next()) return r.fail("missing optical surface line");
    const auto f = tab_fields(r.line);
    if (f.size() < 15) return r.fail("too few fields for an optical surface");
    const char dist = f[1].empty() ? 'g' : f[1][0];
    const int apgr = atoi(f[2].c_str()), optnum = atoi(f[3].c_str()), order = atoi(f[4].c_str());
    const double refl = num_or0(f[5]), trans = num_or0(f[6]), slope = num_or0(f[7]), spec = num_or0(f[8]);
    const double nre = num_or0(f[9]), nim = num_or0(f[10]);
    double grating[4] = {num_or0(f[11]), num_or0(f[12]), num_or0(f[13]), num_or0(f[14])};
    bool use_rt = false, use_tt = false;
    int nr = 0, nt = 0;
    if (f.size() >= 17) {
        use_rt = atoi(f[15].c_str()) > 0;
        nr = atoi(f[16].c_str());
        if (f.size() >= 19) {
            use_tt = atoi(f[17].c_str()) > 0;
            nt = atoi(f[18].c_str());
        }
    }
    std::vector<double> ra, rv, ta, tv;
    if (use_rt && !read_table(r, nr, ra, rv)) return false;
    if (use_tt && !read_table(r, nt, ta, tv)) return false;
    double zero = 0.0;
    if (st_optic(r.ctx, st_uint_t(iopt), fb, dist, optnum, apgr, order, nre, nim, refl, trans, grating, slope, spec,
                 use_rt ? 1 : 0, use_rt ? nr : 0, use_rt ? ra.data() : &zero, use_rt ? rv.data() : &zero,
                 use_tt ? 1 : 0, use_tt ? nt : 0, use_tt ? ta.data() : &zero, use_tt ? tv.data() : &zero) < 0)
        return r.fail("st_optic failed");
    return true;
}

bool read_optics(Reader &r) {
    if (!r.next()) return r.fail("missing OPTICS LIST COUNT");
    int n = 0;
    if (!count_after(r.line, "OPTICS LIST COUNT", n)) return r.fail("expected OPTICS LIST COUNT");
    st_clear_optics(r.ctx);
    for (int i = 0; i < n; ++i) {
        if (!r.next() || r.line.compare(0, 12, "OPTICAL PAIR") != 0) return r.fail("expected OPTICAL PAIR");
        const std::string name = r.line.size() > 13 ? r.line.substr(13) : std::string();
        const int iopt = st_add_optic(r.ctx, name.c_str());
        if (iopt < 0) return r.fail("st_add_optic failed");
        if (!read_face(r, iopt, 1) || !read_face(r, iopt, 2)) return false;
    }
    return true;
}

bool read_element(Reader &r, int stage) {
    if (!r.next()) return r.fail("missing element line");
    const auto f = tab_fields(r.line);
    if (f.size() < 29) return r.fail("too few fields for an element");
    const int e = st_add_element(r.ctx, st_uint_t(stage));
    if (e < 0) return r.fail("st_add_element failed");
    const st_uint_t s = st_uint_t(stage), i = st_uint_t(e);
    st_element_enabled(r.ctx, s, i, atoi(f[0].c_str()) ? 1 : 0);
    st_element_xyz(r.ctx, s, i, num_or0(f[1]), num_or0(f[2]), num_or0(f[3]));
    st_element_aim(r.ctx, s, i, num_or0(f[4]), num_or0(f[5]), num_or0(f[6]));
    st_element_zrot(r.ctx, s, i, num_or0(f[7]));
    if (!f[8].empty()) st_element_aperture(r.ctx, s, i, f[8][0]);
    double p[8];
    for (int k = 0; k < 8; ++k) p[k] = num_or0(f[9 + k]);
    st_element_aperture_params(r.ctx, s, i, p);
    if (!f[17].empty()) st_element_surface(r.ctx, s, i, f[17][0]);
    for (int k = 0; k < 8; ++k) p[k] = num_or0(f[18 + k]);
    if (!f[26].empty()) {
        if (st_element_surface_file(r.ctx, s, i, f[26].c_str()) < 0) return r.fail("cannot read surface file " + f[26]);
    } else {
        st_element_surface_params(r.ctx, s, i, p);
    }
    st_element_optic(r.ctx, s, i, f[27].c_str());
    st_element_interaction(r.ctx, s, i, atoi(f[28].c_str()));
    return true;
}

bool read_stages(Reader &r) {
    if (!r.next()) return r.fail("missing STAGE LIST COUNT");
    int n = 0;
    if (!count_after(r.line, "STAGE LIST COUNT", n)) return r.fail("expected STAGE LIST COUNT");
    st_clear_stages(r.ctx);
    for (int k = 0; k < n; ++k) {
        if (!r.next()) return r.fail("missing STAGE line");
        const auto w = words(r.line);
        if (w.empty() || w[0] != "STAGE") return r.fail("expected STAGE");
        double xyz[3] = {0, 0, 0}, aim[3] = {0, 0, 0}, zrot = 0, virt = 0, multi = 1, count = 0, tt = 0;
        for (size_t i = 0; i + 3 < w.size(); ++i) {
            if (w[i] == "XYZ")
                for (int q = 0; q < 3; ++q) num(w[i + 1 + q], xyz[q]);
            if (w[i] == "AIM")
                for (int q = 0; q < 3; ++q) num(w[i + 1 + q], aim[q]);
        }
        keyed(w, "ZROT", zrot);
        keyed(w, "VIRTUAL", virt);
        keyed(w, "MULTIHIT", multi);
        keyed(w, "ELEMENTS", count);
        keyed(w, "TRACETHROUGH", tt);
        if (!r.next()) return r.fail("missing stage name line");
        const int s = st_add_stage(r.ctx);
        if (s < 0) return r.fail("st_add_stage failed");
        st_stage_flags(r.ctx, st_uint_t(s), int(virt), int(multi), int(tt));
        st_stage_xyz(r.ctx, st_uint_t(s), xyz[0], xyz[1], xyz[2]);
        st_stage_aim(r.ctx, st_uint_t(s), aim[0], aim[1], aim[2]);
        st_stage_zrot(r.ctx, st_uint_t(s), zrot);
        st_clear_elements(r.ctx, st_uint_t(s));
        for (int e = 0; e < int(count); ++e)
            if (!read_element(r, s)) return false;
    }
    return true;
}

// one record value as the CLI prints it: 15 wide, scientific with 6 digits
void put_real(std::string &out, double v) {
    char b[64];
    snprintf(b, sizeof b, "%15.6e", v);
    out += b;
}
void put_int(std::string &out, int v) {
    char b[32];
    snprintf(b, sizeof b, "%15d", v);
    out += b;
}

}  // namespace

extern "C" int st_b200_load_stinput(st_context_t ctx, const char *path) {
    if (!ctx || !path) return -1;
    Reader r;
    r.ctx = ctx;
    r.fp = fopen(path, "r");
    if (!r.fp) {
        st_input_report(ctx, (std::string("cannot open ") + path).c_str());
        return -1;
    }
    bool ok = r.next() && !r.line.empty() && r.line[0] == '#';
    if (!ok) r.fail("the file must start with '# SOLTRACE VERSION x.y.z INPUT FILE'");
    ok = ok && read_sun(r) && read_optics(r) && read_stages(r);
    fclose(r.fp);
    return ok ? 1 : -1;
}

extern "C" int st_b200_write_rays(st_context_t ctx, const char *path) {
    if (!ctx || !path) return -1;
    double x0 = 0, x1 = 0, y0 = 0, y1 = 0;
    int nsun = 0;
    st_sun_stats(ctx, &x0, &x1, &y0, &y1, &nsun);
    const int n = st_num_intersections(ctx);
    if (n < 0) return -1;
    std::vector<double> X(size_t(n) + 1), Y(size_t(n) + 1), Z(size_t(n) + 1), U(size_t(n) + 1), V(size_t(n) + 1),
        W(size_t(n) + 1);
    std::vector<int> em(size_t(n) + 1), sm(size_t(n) + 1), rn(size_t(n) + 1);
    if (n > 0 && (st_locations(ctx, X.data(), Y.data(), Z.data()) < 0 || st_cosines(ctx, U.data(), V.data(), W.data()) < 0 ||
                  st_elementmap(ctx, em.data()) < 0 || st_stagemap(ctx, sm.data()) < 0 ||
                  st_raynumbers(ctx, rn.data()) < 0))
        return -1;
    FILE *fp = fopen(path, "w");
    if (!fp) {
        st_input_report(ctx, (std::string("cannot write ") + path).c_str());
        return -1;
    }
    std::string out;
    out.reserve(size_t(n) * 136 + 512);
    out += "#       SunXMin        SunXMax        SunYMin        SunYMax    SunRayCount         Length\n";
    for (double v : {x0, x1, y0, y1, double(nsun), double(n)}) put_real(out, v);
    out += "\n";
    out += "#             X              Y              Z           Xcos           Ycos           Zcos       Stagemap     "
           "Elementmap      Raynumber\n";
    for (int i = 0; i < n; ++i) {
        put_real(out, X[i]);
        put_real(out, Y[i]);
        put_real(out, Z[i]);
        put_real(out, U[i]);
        put_real(out, V[i]);
        put_real(out, W[i]);
        put_int(out, sm[i]);
        put_int(out, em[i]);
        put_int(out, rn[i]);
        out += "\n";
        if (out.size() > (size_t(1) << 24)) {
            fwrite(out.data(), 1, out.size(), fp);
            out.clear();
        }
    }
    const bool ok = fwrite(out.data(), 1, out.size(), fp) == out.size();
    return (fclose(fp) == 0 && ok) ? 1 : -1;
}
