// Prints the coordinate maps of the drop-in's symmetry operations (Tnm,
// Tnm_general, sigma_n_arb, GetElemProd) and the group element arrays that
// SymmetryClass builds from them, one line per case:
//   <case> <n> x0 y0 x1 y1 ...          transformed coordinates
//   <case>_perm <n> p0 p1 ...           element array (reference layout)
// Sites are listed as the reference's examples create them (i over a1
// outermost, j over a2).  Host code only: no GPU is needed.
#include <cmath>
#include <cstdio>
#include <vector>

#include "qmb/qmbcuda.hpp"

static void sites(const LatticeGeometryInfo& g, float x0, float y0, std::vector<float>& R1, std::vector<float>& R2) {
    R1.clear();
    R2.clear();
    for (int i = 0; i < g.N1; ++i)
        for (int j = 0; j < g.N2; ++j) {
            R1.push_back(i * g.A_mat[0][0] + j * g.A_mat[0][1] + x0);
            R2.push_back(i * g.A_mat[1][0] + j * g.A_mat[1][1] + y0);
        }
}

static void print_map(const char* name, SiteMap m, const std::vector<float>& R1, const std::vector<float>& R2) {
    std::vector<float> a, b;
    m(R1, R2, a, b);
    std::printf("%s %zu", name, a.size());
    for (size_t i = 0; i < a.size(); ++i) std::printf(" %.7g %.7g", a[i], b[i]);
    std::printf("\n");
    std::vector<std::vector<qmb_complex>> ch = {{qmb_complex(1.0f, 0.0f)}};
    SymmetryClass<qmb_complex> G(ch, std::vector<SiteMap>{m});
    std::vector<uint32_t> p(R1.size());
    G.GetGroupElemArr(R1, R2, p.data());
    std::printf("%s_perm %zu", name, p.size());
    for (uint32_t v : p) std::printf(" %u", v);
    std::printf("\n");
}

int main() {
    std::vector<float> R1, R2;
    LatticeGeometryInfo sq46 = create_square_lattice_info(4, 6);
    sites(sq46, 0.0f, 0.0f, R1, R2);
    print_map("tnm_square_4x6_11", Tnm(4, 6, 1, 1), R1, R2);
    print_map("tnm_general_square_4x6_11", Tnm_general(1, 1, sq46), R1, R2);
    LatticeGeometryInfo tri46 = create_triangular_lattice_info(4, 6);
    sites(tri46, 0.0f, 0.0f, R1, R2);
    print_map("tnm_general_triangular_4x6_11", Tnm_general(1, 1, tri46), R1, R2);
    print_map("tnm_general_triangular_4x6_32", Tnm_general(3, 2, tri46), R1, R2);
    LatticeGeometryInfo sq64 = create_square_lattice_info(6, 4);
    sites(sq64, 0.0f, 0.0f, R1, R2);
    print_map("tnm_general_square_6x4_14", Tnm_general(1, 4, sq64), R1, R2);
    // reflections of a 4x4 square lattice centred on the origin
    LatticeGeometryInfo sq44 = create_square_lattice_info(4, 4);
    sites(sq44, -1.5f, -1.5f, R1, R2);
    print_map("sigma_0", sigma_n_arb(0.0f), R1, R2);
    print_map("sigma_45", sigma_n_arb(45.0f), R1, R2);
    print_map("sigma_90", sigma_n_arb(90.0f), R1, R2);
    print_map("sigma_135", sigma_n_arb(135.0f), R1, R2);
    print_map("prod_sigma_0_sigma_90", GetElemProd(sigma_n_arb(0.0f), sigma_n_arb(90.0f)), R1, R2);
    print_map("prod_sigma_0_c4", GetElemProd(sigma_n_arb(0.0f), Cn(4, {0.0f, 0.0f})), R1, R2);
    return 0;
}
