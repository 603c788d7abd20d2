// The reference's own known-answer tests (test_ILU0_mod.pf, test_ILU0_HB_mod.pf,
// test_fgmres.pf, test_fgmres_ref.pf), replayed through the C++ host layer
// (include/chidg_gpu.hpp) in the reference's terms: a chidg_matrix_t of 1 x 1
// blocks poked block by block, create_preconditioner('ilu0') / ('identity'),
// create_linear_solver('fgmres'), and the asserted LD entries, z and x.
//
// Input: the cases of tests/golden/reference_kat.json as text lines
//   case <name> <nelem_xi> <ntime> <tol> <solver_tol>
//   block <elem> <time> <col_elem> <value>      (1-based ids, LOCAL blocks)
//   rhs <elem> <value>
//   LD <elem> <time> <col_elem> <value> | z <elem> <entry> <value> | x <elem> <entry> <value>
//   end
// Exit status 0 when every assert holds.
#include "chidg_gpu.hpp"

#include <cmath>
#include <cstdio>
#include <fstream>
#include <sstream>
#include <string>
#include <tuple>
#include <vector>

using namespace chidg_gpu;

struct Case {
    std::string name;
    int nelem_xi = 0, ntime = 1;
    double tol = 0, solver_tol = 0;
    std::vector<std::tuple<int, int, int, double>> blocks, ld_asserts;
    std::vector<std::pair<int, double>> rhs;
    std::vector<std::tuple<char, int, int, double>> vec_asserts;   // 'z' or 'x'
};

static int failures = 0;
static void expect(bool ok, const std::string& what) {
    if (!ok) { std::printf("FAIL %s\n", what.c_str()); ++failures; }
}

// packed position of the LOCAL 1 x 1 block (row e, time t, column c), 1-based ids
static int64_t ld_index(const Pattern& p, int e, int t, int c) {
    for (int64_t k = 0; k < p.nblocks(); ++k)
        if (p.blk_kind[k] == CHIDG_BLK_LOCAL && p.blk_row_elem[k] == e - 1 && p.blk_row_time[k] == t - 1 &&
            p.blk_col_elem[k] == c - 1)
            return k;
    return -1;
}

static void run(Context& ctx, const Case& cs) {
    const Pattern pat = Pattern::box(cs.nelem_xi, 1, 1, 1, 1, cs.ntime);
    ChidgMatrix A(ctx, pat);
    std::vector<double> vals((size_t)A.nvalues(), 0.0);
    for (const auto& [e, t, c, v] : cs.blocks) {
        const int64_t k = ld_index(pat, e, t, c);
        expect(k >= 0, cs.name + ": block in the pattern");
        if (k >= 0) vals[(size_t)k] = v;
    }
    A.store(vals);
    std::vector<double> b((size_t)A.nvec(), 0.0);
    for (const auto& [e, v] : cs.rhs)
        for (int t = 0; t < cs.ntime; ++t) b[(size_t)((e - 1) * cs.ntime + t)] = v;
    ChidgVector rhs(A, b);
    if (cs.name.rfind("ilu0", 0) == 0) {
        auto M = create_preconditioner("ILU0");
        M->update(A, &rhs);
        const std::vector<double> LD = M->LD();
        for (const auto& [e, t, c, v] : cs.ld_asserts) {
            const int64_t k = ld_index(pat, e, t, c);
            expect(k >= 0 && LD[(size_t)k] == v, cs.name + ": LD(" + std::to_string(e) + "," + std::to_string(c) + ")");
        }
        const std::vector<double> z = M->apply(A, rhs).get();
        for (const auto& [kind, e, i, v] : cs.vec_asserts)
            if (kind == 'z')
                expect(std::fabs(z[(size_t)((e - 1) * cs.ntime + i - 1)] - v) <= cs.tol, cs.name + ": z(" + std::to_string(e) + ")");
    } else {
        auto M = create_preconditioner("identity");
        auto solver = create_linear_solver("fgmres");
        solver->set("tol", cs.solver_tol);     // linear_solver%tol as the test sets it
        solver->set("nmax", 1000.0);
        ChidgVector x(A);
        solver->solve(A, x, rhs, *M);
        const std::vector<double> xv = x.get();
        for (const auto& [kind, e, i, v] : cs.vec_asserts)
            if (kind == 'x')
                expect(std::fabs(xv[(size_t)((e - 1) * cs.ntime + i - 1)] - v) <= cs.tol, cs.name + ": x(" + std::to_string(e) + ")");
        expect(solver->residual_norm < 1e-12, cs.name + ": true residual");
    }
    std::printf("%s: done\n", cs.name.c_str());
}

int main(int argc, char** argv) {
    if (argc < 2) { std::printf("usage: %s cases.txt\n", argv[0]); return 2; }
    std::ifstream in(argv[1]);
    std::vector<Case> cases;
    std::string line;
    Case cur;
    while (std::getline(in, line)) {
        std::istringstream ls(line);
        std::string tag;
        ls >> tag;
        if (tag == "case") ls >> cur.name >> cur.nelem_xi >> cur.ntime >> cur.tol >> cur.solver_tol;
        else if (tag == "block") { int e, t, c; double v; ls >> e >> t >> c >> v; cur.blocks.emplace_back(e, t, c, v); }
        else if (tag == "rhs") { int e; double v; ls >> e >> v; cur.rhs.emplace_back(e, v); }
        else if (tag == "LD") { int e, t, c; double v; ls >> e >> t >> c >> v; cur.ld_asserts.emplace_back(e, t, c, v); }
        else if (tag == "z" || tag == "x") { int e, i; double v; ls >> e >> i >> v; cur.vec_asserts.emplace_back(tag[0], e, i, v); }
        else if (tag == "end") { cases.push_back(cur); cur = Case(); }
    }
    try {
        Context ctx(0);
        for (const Case& cs : cases) run(ctx, cs);
        // the factory refuses unknown names, as create_preconditioner signals FATAL
        bool threw = false;
        try { create_preconditioner("ilu1"); } catch (const Error& e) { threw = e.code == CHIDG_GPU_EINVAL; }
        expect(threw, "create_preconditioner('ilu1') refused");
    } catch (const Error& e) {
        std::printf("FAIL exception %d: %s\n", e.code, e.what());
        return 1;
    }
    std::printf("%d cases, %d failures\n", (int)cases.size(), failures);
    return failures == 0 ? 0 : 1;
}
