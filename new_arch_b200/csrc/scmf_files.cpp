// Reference file surface of libscmf: configuration.dat / polymer.dat parsers,
// density_<step>.dat and coord.dat writers, the coord.dat reader and the VTK
// converter.  Formats follow the reference byte for byte; the parsers use the
// same literal scanf patterns (init_config.cu:214-340, 491-512) because the
// input files are defined by them.
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <vector>

#include "scmf_engine.h"

using namespace scmf;

namespace {

struct File {
    FILE* f = nullptr;
    explicit File(FILE* p) : f(p) {}
    ~File() {
        if (f) fclose(f);
    }
};

}  // namespace

extern "C" {

// configuration.dat (init_config.cu:487-512) + polymer.dat (init_config.cu:214-340).
// Derived constants: harmonic_normb = 1/(2 sigma^2), sigma = 1/sqrt(3(N_ref-1))
// (init_config.cu:480-484); A = dt*N/xi / N_ref, R = sqrt(2A) (init_config.cu:807-808);
// initial per-component bond sigma 1/sqrt(3(length-1)) per architecture
// (device_function.cu:169-171); SCMF0 field, omega skipped when step % 10 == 0.
scmf_status scmf_spec_load_files(const char* cfg_path, const char* poly_path, uint64_t seed, scmf_spec** out) {
    if (!cfg_path || !poly_path || !out) return fail(SCMF_E_INVALID, "NULL argument");
    *out = nullptr;
    // polymer.dat first, as the reference does (Read_polymer_config precedes initialize_values)
    File pf(fopen(poly_path, "r"));
    if (!pf.f) return fail(SCMF_E_IO, "cannot open %s: %s", poly_path, strerror(errno));
    int n_ptypes = 0, n_polymers = 0;
    if (fscanf(pf.f, "Number of polymer type:%d\n", &n_ptypes) != 1 || n_ptypes < 1 || n_ptypes > 64)
        return fail(SCMF_E_PARSE, "%s: bad 'Number of polymer type:' line", poly_path);
    if (fscanf(pf.f, "Number of total polymer:%d\n", &n_polymers) != 1 || n_polymers < 0)
        return fail(SCMF_E_PARSE, "%s: bad 'Number of total polymer:' line", poly_path);
    std::vector<int> per_type(n_ptypes);
    long long sum = 0;
    for (int i = 0; i < n_ptypes; ++i) {
        if (fscanf(pf.f, "%d ", &per_type[i]) != 1 || per_type[i] < 0)
            return fail(SCMF_E_PARSE, "%s: bad per-type polymer count %d", poly_path, i);
        sum += per_type[i];
    }
    if (sum != n_polymers) return fail(SCMF_E_PARSE, "%s: per-type counts sum to %lld, total says %d", poly_path, sum, n_polymers);
    if (fscanf(pf.f, "\n--------\n") != 0) return fail(SCMF_E_PARSE, "%s: missing separator", poly_path);
    int nref = 0;
    std::vector<scmf_spec::Arch> archs;
    for (int p = 0; p < n_ptypes; ++p) {
        int tmp = 0, L = 0;
        if (fscanf(pf.f, "Polymer type: %d\n", &tmp) != 1) return fail(SCMF_E_PARSE, "%s: bad 'Polymer type:' (%d)", poly_path, p);
        if (fscanf(pf.f, "Polymer length: %d\n", &L) != 1 || L < 1 || L > kMaxLength)
            return fail(SCMF_E_PARSE, "%s: bad 'Polymer length:' (%d)", poly_path, p);
        if (fscanf(pf.f, "Polymer length unit: %d\n", &nref) != 1 || nref < 2)
            return fail(SCMF_E_PARSE, "%s: bad 'Polymer length unit:' (%d)", poly_path, p);
        if (fscanf(pf.f, "Monomer type: ") != 0) return fail(SCMF_E_PARSE, "%s: missing 'Monomer type:'", poly_path);
        scmf_spec::Arch a;
        a.length = L;
        a.n_chains = per_type[p];
        a.type.resize(L);
        for (int i = 0; i < L; ++i)
            if (fscanf(pf.f, "%d ", &a.type[i]) != 1) return fail(SCMF_E_PARSE, "%s: bad monomer type list", poly_path);
        fscanf(pf.f, "\n");
        // connection matrix: row i, column j; conection_list[i] = {j : row i has 1 at column j}
        for (int i = 0; i < L; ++i) {
            for (int j = 0; j < L; ++j) {
                int v = 0;
                if (fscanf(pf.f, "%d ", &v) != 1) return fail(SCMF_E_PARSE, "%s: bad connection matrix", poly_path);
                if (v == 1 && j > i) {
                    a.bonds.push_back(i);
                    a.bonds.push_back(j);
                } else if (v == 1 && j < i) {
                    // symmetric matrices (all reference inputs) contribute each bond once
                    bool seen = false;
                    for (size_t b = 0; b + 1 < a.bonds.size(); b += 2)
                        if (a.bonds[b] == j && a.bonds[b + 1] == i) seen = true;
                    if (!seen) {
                        a.bonds.push_back(j);
                        a.bonds.push_back(i);
                    }
                }
            }
            fscanf(pf.f, "\n");
        }
        a.init_sigma = L > 1 ? 1.0 / std::sqrt(3.0 * (L - 1.0)) : 0.0;
        archs.push_back(std::move(a));
    }

    File cf(fopen(cfg_path, "r"));
    if (!cf.f) return fail(SCMF_E_IO, "cannot open %s: %s", cfg_path, strerror(errno));
    int n = 0;
    if (fscanf(cf.f, "Monomer type number: %d\n", &n) != 1 || n < 1 || n > kMaxTypes)
        return fail(SCMF_E_PARSE, "%s: bad 'Monomer type number:' line", cfg_path);
    std::vector<double> xn((size_t)n * n);
    for (int j = 0; j < n; ++j) {
        for (int i = 0; i < n; ++i)
            if (fscanf(cf.f, "%lg ", &xn[(size_t)i + (size_t)n * j]) != 1)
                return fail(SCMF_E_PARSE, "%s: bad interaction matrix", cfg_path);
        fscanf(cf.f, "\n");
    }
    double lx = 0, ly = 0, lz = 0, xiN = 0, dtNxi = 0, kT = 0;
    int nx = 0, ny = 0, nz = 0, time0 = 0;
    if (fscanf(cf.f, "D0 =     %lg; LY =    %lg; LZ =    %lg;\n", &lx, &ly, &lz) != 3)
        return fail(SCMF_E_PARSE, "%s: bad 'D0 = ; LY = ; LZ = ;' line", cfg_path);
    if (fscanf(cf.f, "N = %d %d %d \n", &nx, &ny, &nz) != 3) return fail(SCMF_E_PARSE, "%s: bad 'N =' line", cfg_path);
    if (fscanf(cf.f, "time =  %d;\n", &time0) != 1) return fail(SCMF_E_PARSE, "%s: bad 'time =' line", cfg_path);
    if (fscanf(cf.f, "xiN = %lg;\n", &xiN) != 1) return fail(SCMF_E_PARSE, "%s: bad 'xiN =' line", cfg_path);
    if (fscanf(cf.f, "dt*N/xi = %lg;\n", &dtNxi) != 1) return fail(SCMF_E_PARSE, "%s: bad 'dt*N/xi =' line", cfg_path);
    if (fscanf(cf.f, "kT = %lg;\n", &kT) != 1) return fail(SCMF_E_PARSE, "%s: bad 'kT =' line", cfg_path);

    for (const auto& a : archs)
        for (int t : a.type)
            if (t < 0 || t >= n) return fail(SCMF_E_PARSE, "%s: monomer type %d but %s declares %d types", poly_path, t, cfg_path, n);

    std::unique_ptr<scmf_spec> s(new scmf_spec);
    s->n_types = n;
    s->nx = nx; s->ny = ny; s->nz = nz;
    s->lx = lx; s->ly = ly; s->lz = lz;
    s->xn = xn;
    s->archs = std::move(archs);
    const double sigma = 1.0 / std::sqrt(3.0 * (nref - 1.0));
    s->p.reference_nbeads = nref;
    s->p.harmonic_normb = 1.0 / (2.0 * sigma * sigma);
    s->p.smc_a = dtNxi / nref;
    s->p.seed = seed;
    s->p.hamiltonian = SCMF_HAM_SCMF0;
    s->p.field_rule = SCMF_FIELD_REFERENCE;
    s->p.count_bits = 32;
    scmf_status rc = validate_spec(*s);
    if (rc) return rc;
    *out = s.release();
    return SCMF_OK;
}

// density_<step>.dat (io.cpp:4-56): header, then per cell the n_types volume
// fractions count * n_cells / n_beads and the n_types omega values, "%g ".
scmf_status scmf_write_density(const scmf_system* s, const char* path, int64_t step) {
    if (!s) return fail(SCMF_E_INVALID, "NULL system");
    const int n = s->spec.n_types;
    const size_t nc = (size_t)s->n_cells;
    std::vector<uint32_t> cnt(nc * n);
    std::vector<float> om(nc * n);
    scmf_status rc = scmf_get_counts(s, cnt.data(), cnt.size());
    if (rc) return rc;
    if ((rc = scmf_get_omega(s, om.data(), om.size()))) return rc;
    char name[64];
    if (!path) {
        if (step < 1000000)
            snprintf(name, sizeof name, "density_%d.dat", (int)step);
        else
            snprintf(name, sizeof name, "density_%ge+06.dat", (double)step / 1000000);
        path = name;
    }
    FILE* f = fopen(path, "w");
    if (!f) return fail(SCMF_E_IO, "cannot open %s: %s", path, strerror(errno));
    const double scale = (double)nc / (double)s->n_beads;
    fprintf(f, "Nx=%d, Ny=%d, Nz=%d\n", s->spec.nx, s->spec.ny, s->spec.nz);
    fprintf(f, "dx=%g, dy=%g, dz=%g\n", s->spec.lx / s->spec.nx, s->spec.ly / s->spec.ny, s->spec.lz / s->spec.nz);
    for (size_t c = 0; c < nc; ++c) {
        for (int t = 0; t < n; ++t) fprintf(f, "%g ", (int)cnt[c + t * nc] * scale);
        for (int t = 0; t < n; ++t) fprintf(f, "%g ", (double)om[c + t * nc]);
        fprintf(f, "\n");
    }
    if (fclose(f) != 0) return fail(SCMF_E_IO, "write to %s failed", path);
    return SCMF_OK;
}

// coord.dat (io.cpp:95-118): "%g %g %g\n" per bead, unwrapped coordinates.
scmf_status scmf_write_coords(const scmf_system* s, const char* path) {
    if (!s || !path) return fail(SCMF_E_INVALID, "NULL argument");
    std::vector<float> xyz((size_t)s->n_beads * 3);
    scmf_status rc = scmf_get_coords(s, xyz.data(), xyz.size());
    if (rc) return rc;
    FILE* f = fopen(path, "w");
    if (!f) return fail(SCMF_E_IO, "cannot open %s: %s", path, strerror(errno));
    for (int64_t i = 0; i < s->n_beads; ++i)
        fprintf(f, "%g %g %g\n", (double)xyz[3 * i], (double)xyz[3 * i + 1], (double)xyz[3 * i + 2]);
    if (fclose(f) != 0) return fail(SCMF_E_IO, "write to %s failed", path);
    return SCMF_OK;
}

// coord.dat reader (init_config.cu:951-980).
scmf_status scmf_read_coords_file(const char* path, int64_t skip, float* xyz, size_t n) {
    if (!path || !xyz || n % 3 != 0 || skip < 0) return fail(SCMF_E_INVALID, "bad arguments");
    File f(fopen(path, "r"));
    if (!f.f) return fail(SCMF_E_IO, "cannot open %s: %s", path, strerror(errno));
    double a, b, c;
    for (int64_t i = 0; i < skip; ++i)
        if (fscanf(f.f, "%lg %lg %lg\n", &a, &b, &c) != 3) return fail(SCMF_E_PARSE, "%s: short file at line %lld", path, (long long)i + 1);
    for (size_t i = 0; i < n / 3; ++i) {
        if (fscanf(f.f, "%lg %lg %lg\n", &a, &b, &c) != 3)
            return fail(SCMF_E_PARSE, "%s: short file at line %lld", path, (long long)(skip + (int64_t)i + 1));
        xyz[3 * i] = (float)a;
        xyz[3 * i + 1] = (float)b;
        xyz[3 * i + 2] = (float)c;
    }
    return SCMF_OK;
}

// vtk.c:4-81: STRUCTURED_POINTS of phi_0 - phi_1, "%7.4lf " per point, one
// line per (y, z) row.  vtk.c reads six numbers per grid point whatever the
// file holds; values_per_point = 6 keeps that behaviour, 0 derives the count
// (2 * n_types) from the first data line.
scmf_status scmf_vtk_convert(const char* in, const char* out, int32_t vpp) {
    if (!in || !out || vpp < 0 || vpp > 2 * kMaxTypes + 64) return fail(SCMF_E_INVALID, "bad arguments");
    File fp(fopen(in, "r"));
    if (!fp.f) return fail(SCMF_E_IO, "cannot open %s", in);
    int Nx = 0, Ny = 0, Nz = 0;
    double dx = 0, dy = 0, dz = 0;
    if (fscanf(fp.f, "Nx=%d, Ny=%d, Nz=%d\n", &Nx, &Ny, &Nz) != 3 || Nx < 1 || Ny < 1 || Nz < 1)
        return fail(SCMF_E_PARSE, "%s: bad 'Nx=' header", in);
    if (fscanf(fp.f, "dx=%lf, dy=%lf, dz=%lf\n", &dx, &dy, &dz) != 3) return fail(SCMF_E_PARSE, "%s: bad 'dx=' header", in);
    if (vpp == 0) {
        long pos = ftell(fp.f);
        char line[4096];
        if (!fgets(line, sizeof line, fp.f)) return fail(SCMF_E_PARSE, "%s: no data", in);
        int cnt = 0;
        char* p = line;
        for (;;) {
            char* e = nullptr;
            strtod(p, &e);
            if (e == p) break;
            ++cnt;
            p = e;
        }
        fseek(fp.f, pos, SEEK_SET);
        vpp = cnt;
        if (vpp < 2) return fail(SCMF_E_PARSE, "%s: fewer than two values per point", in);
    }
    FILE* fw = fopen(out, "w");
    if (!fw) return fail(SCMF_E_IO, "cannot open %s", out);
    fprintf(fw, "# vtk DataFile Version 3.0\n");
    fprintf(fw, "# comment: converted from file %s\n", in);
    fprintf(fw, "ASCII\n");
    fprintf(fw, "DATASET STRUCTURED_POINTS\n");
    fprintf(fw, "DIMENSIONS %d %d %d\n", Nx, Ny, Nz);
    fprintf(fw, "ORIGIN 0.000000 0.000000 0.000000\n");
    fprintf(fw, "SPACING %.6lf %.6lf %.6lf\n\n", dx, dy, dz);
    fprintf(fw, "POINT_DATA %ld\n", (long)Nx * Ny * Nz);
    fprintf(fw, "SCALARS scalars float\n");
    fprintf(fw, "LOOKUP_TABLE default\n\n");
    std::vector<double> v((size_t)vpp, 0.0);
    for (int k = 0; k < Nz; ++k)
        for (int j = 0; j < Ny; ++j) {
            for (int i = 0; i < Nx; ++i) {
                // a short read leaves the remaining values as they were, like fscanf
                for (int q = 0; q < vpp; ++q)
                    if (fscanf(fp.f, "%lf", &v[q]) != 1) break;
                fprintf(fw, "%7.4lf ", v[0] - v[1]);
            }
            fprintf(fw, "\n");
        }
    if (fclose(fw) != 0) return fail(SCMF_E_IO, "write to %s failed", out);
    return SCMF_OK;
}

}  // extern "C"
