// Known-answer checks of the C++ facade (include/paulib_b200.hpp) on the GPU,
// restating assertions of the reference's tests/PauliSumTests.cpp (lines
// cited per check).  Prints one line per failure; exit status 0 when all
// pass.
#include <cmath>
#include <cstdio>
#include <map>
#include <string>
#include <utility>
#include <vector>

#include "paulib_b200.hpp"

using paulib_b200::PauliSum;
using paulib_b200::TruncationOptions;
using Terms = std::vector<std::pair<std::string, double>>;  // as the reference's tests spell it

static int g_fail = 0, g_pass = 0;
#define EXPECT(cond)                                                          \
    do {                                                                      \
        if (cond) {                                                           \
            ++g_pass;                                                         \
        } else {                                                              \
            ++g_fail;                                                         \
            std::printf("FAIL %s:%d: %s\n", __FILE__, __LINE__, #cond);       \
        }                                                                     \
    } while (0)

template <std::size_t N>
static std::map<std::string, double> terms(PauliSum<N>& s) {
    std::map<std::string, double> out;
    const std::string str = s.get_str();
    std::size_t pos = 0;
    while (pos < str.size()) {
        const std::size_t eol = str.find('\n', pos);
        const std::string line = str.substr(pos, eol - pos);
        const std::size_t star = line.find(" * ");
        out[line.substr(star + 3)] = std::stod(line.substr(0, star));
        pos = eol + 1;
    }
    return out;
}

int main() {
    // :397-414 Cayley table with phases (X*Y = iZ, Y*X = -iZ)
    {
        PauliSum<1> a(Terms{{"X", 1.0}}), b(Terms{{"Y", 1.0}});
        PauliSum<1> c = a * b;
        EXPECT(c.get_str() == "1.000000 * iZ\n");
        PauliSum<1> d = b * a;
        EXPECT(d.get_str() == "1.000000 * -iZ\n");
    }
    // :514-561 sort_and_combine merges equal keys, keeps the sign in the key
    {
        PauliSum<2> s(Terms{{"XY", 2.0}, {"ZZ", 1.0}, {"XY", 3.0}});
        s.sort_and_combine();
        EXPECT(s.get_str() == "1.000000 * ZZ\n5.000000 * XY\n");
        PauliSum<1> t(Terms{{"X", 2.0}, {"-X", 3.0}});
        t.sort_and_combine();
        EXPECT(t.get_length() == 2);
    }
    // :567-646 `+=` appends then combines
    {
        PauliSum<2> a(Terms{{"XX", 1.0}, {"ZZ", 2.0}}), b(Terms{{"XX", 3.0}});
        a += b;
        EXPECT(a.get_str() == "2.000000 * ZZ\n4.000000 * XX\n");
    }
    // :1075-1111 canonicalize folds the sign, drops zeros, keeps the phase bit
    {
        PauliSum<2> s(Terms{{"XI", 1.0}, {"-XI", 0.25}, {"ZI", 2.0}});
        s.canonicalize();
        auto m = terms(s);
        EXPECT(m.size() == 2 && m["XI"] == 0.75 && m["ZI"] == 2.0);
        PauliSum<1> z(Terms{{"-iZ", 3.0}});
        z.canonicalize();
        EXPECT(z.get_str() == "-3.000000 * iZ\n");
    }
    // :1113-1137 trim and trim with a keep set
    {
        PauliSum<2> s(Terms{{"XI", 0.1}, {"ZI", -5.0}, {"IZ", 0.3}, {"YI", 2.0}});
        s.trim(2);
        auto m = terms(s);
        EXPECT(m.size() == 2 && m["ZI"] == -5.0 && m["YI"] == 2.0);
        PauliSum<2> p(Terms{{"XI", 0.001}, {"ZI", -5.0}, {"IZ", 0.3}, {"YI", 2.0}});
        PauliSum<2> keep(2, "XI", 1.0);
        p.trim(2, keep);
        auto q = terms(p);
        EXPECT(q.size() == 2 && q["XI"] == 0.001 && q["ZI"] == -5.0);
    }
    // :1139-1147 cutoff and truncate_weight
    {
        PauliSum<3> s(Terms{{"XII", 0.5}, {"XYZ", 0.01}, {"ZZI", -0.2}});
        s.cutoff(0.05);
        EXPECT(s.get_length() == 2);
        s.truncate_weight(1);
        EXPECT(s.get_str() == "0.500000 * XII\n");
    }
    // :826-879 CNOT truth table entries
    {
        PauliSum<2> s(Terms{{"XZ", 1.0}});
        s.apply_CNOT(0, 1);
        EXPECT(s.get_str() == "1.000000 * -YY\n");
        PauliSum<2> t(Terms{{"YY", 1.0}});
        t.apply_CNOT(0, 1);
        EXPECT(t.get_str() == "1.000000 * -XZ\n");
    }
    // :899-983 evolve fast paths and the general angle
    {
        PauliSum<1> s(Terms{{"X", 1.0}});
        s.evolve(PauliSum<1>(Terms{{"Z", M_PI / 2}}));
        EXPECT(s.get_str() == "1.000000 * -Y\n");
        PauliSum<1> g(Terms{{"X", 1.0}});
        g.evolve(PauliSum<1>(Terms{{"Z", M_PI / 3}}));
        g.download();
        EXPECT(g.value.size() == 2 && g.value[0] == std::cos(M_PI / 3) &&
               g.value[1] == -std::sin(M_PI / 3));
    }
    // :689-712 zero_state_expectation: only I/Z strings, sign and phase rules
    {
        PauliSum<2> s(Terms{{"II", 1.5}, {"ZI", 2.0}, {"ZZ", 4.0}, {"XI", 8.0}, {"IY", 16.0}});
        EXPECT(s.zero_state_expectation() == 7.5);
    }
    // commutator values: [X, Z] = -2i Y (x 1.5 x 2), i[X, Z] = 2 Y
    {
        PauliSum<1> a(Terms{{"X", 1.5}}), b(Terms{{"Z", 2.0}});
        auto c = paulib_b200::commutator(a, b);
        EXPECT(c.get_str() == "6.000000 * -iY\n");
        auto ic = paulib_b200::i_commutator(a, b);
        EXPECT(ic.get_str() == "6.000000 * Y\n");
    }
    // propagate / propagate_expectation agree with evolve + apply_truncation
    // walked backwards by hand
    {
        PauliSum<4> obs(Terms{{"ZIII", 1.0}, {"IZII", 0.5}});
        PauliSum<4> rot(Terms{{"XIII", 0.3}, {"IYII", 1.1}, {"ZXII", 0.7}, {"IIXI", 2.0}});
        TruncationOptions<double> o;
        o.max_weight = 3;
        o.coefficient_cutoff = 1e-3;
        const double e = paulib_b200::propagate_expectation(obs, rot, o);
        PauliSum<4> h(obs);
        rot.download();
        for (std::size_t r = rot.value.size(); r-- > 0;) {
            PauliSum<4> one(4);
            for (std::size_t k = 0; k < 1; ++k) {
                one.x_data[k] = {rot.x_data[k][r]};
                one.z_data[k] = {rot.z_data[k][r]};
            }
            one.flags = {rot.flags[r]};
            one.value = {rot.value[r]};
            one.upload();
            h.evolve(one);
            h.canonicalize();
            h.truncate_weight(3);
            h.cutoff(1e-3);
        }
        EXPECT(std::fabs(h.zero_state_expectation() - e) <= 1e-12);
    }
    // PauliSumTests.cpp:313-325 and 243-256: H gates and apply_RZ
    {
        PauliSum<4> s(Terms{{"IZXY", 1.0}});
        for (std::size_t q = 0; q < 4; ++q) s.apply_H(q);
        EXPECT(s.get_str() == "1.000000 * -IXZY\n");
        PauliSum<1> r(Terms{{"Z", 2.0}, {"X", 1.0}});
        r.apply_RZ(0, M_PI / 3.0);
        EXPECT(r.get_str() == "2.000000 * Z\n0.866025 * X\n0.500000 * -Y\n");
        PauliSum<2> c(Terms{{"XI", 1.0}});
        c.apply_iSWAP(0, 1);
        EXPECT(c.get_str() == "1.000000 * ZY\n");
    }
    // PauliSumTests.cpp:715-760, 764-816, 1041-1070: reductions
    {
        PauliSum<2> s(Terms{{"ZI", 2.0}, {"IZ", 3.0}, {"ZZ", 4.0}});
        s.canonicalize();
        PauliSum<2> t(Terms{{"ZI", 2.0}, {"IZ", 3.0}, {"ZZ", 4.0}});
        EXPECT(t.basis_state_expectation("10") == -2.0 + 3.0 - 4.0);
        bool threw = false;
        try {
            t.basis_state_expectation("000");
        } catch (const std::invalid_argument&) {
            threw = true;
        }
        EXPECT(threw);
        PauliSum<1> l(Terms{{"X", 1.0}, {"-X", 0.25}, {"iY", 2.0}});
        EXPECT(l.lookup("X") == 0.75 && l.lookup("-iY") == -2.0);
        PauliSum<4> tr(Terms{{"IIII", 2.5}, {"XIZI", 7.0}, {"-IIII", 1.0}, {"iIIII", 3.0}});
        EXPECT(tr.trace() == 16.0 * 1.5);
        PauliSum<3> a(3, "XYZ", 1.0), b(3, "XYI", 1.0);
        EXPECT(paulib_b200::trace_product(a, a) == 8.0 && paulib_b200::trace_product(a, b) == 0.0);
    }
    // errors map to the reference's exception types
    {
        bool threw = false;
        try {
            PauliSum<1> s(Terms{{"XQ", 1.0}});
        } catch (const std::invalid_argument&) {
            threw = true;
        }
        EXPECT(threw);
    }
    std::printf("facade: %d passed, %d failed\n", g_pass, g_fail);
    return g_fail == 0 ? 0 : 1;
}
