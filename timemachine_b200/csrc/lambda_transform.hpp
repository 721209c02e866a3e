// Lambda transforms of the nonbonded potentials: the four schedules
// (charge, sigma, epsilon, w) that the reference constructors take as C++
// expression strings in `lambda` (timemachine/cpp/src/wrap_kernels.cpp:843-893,
// substituted into timemachine/cpp/src/kernels/k_lambda_transformer_jit.cuh:8-22
// and compiled at run time there).
//
// Each schedule is a function of the scalar lambda only, so its value f and
// derivative g = df/dlambda are the same for every atom of a call. Here the
// expression is parsed once on the host and evaluated per call in forward-mode
// dual numbers (value, derivative), and the staging kernels receive (f, g) of
// every window as launch arguments: no run-time compilation, and a call stays
// graph-capturable.
//
// Language: the C expression subset the transforms use -- numeric literals
// (C rules: an integer literal is an int, and int op int is integer arithmetic,
// so "1/2" is 0 as in the reference's compiled code), `lambda`, `PI`, unary
// + - !, binary * / % + - < <= > >= == != && ||, the conditional ?:,
// parentheses, and the functions sin cos tan asin acos atan atan2 sinh cosh
// tanh exp log log10 sqrt pow fabs abs fmin fmax min max floor ceil.
//
// Derivatives are exact (rounded) derivatives of the expression; the reference
// takes them by a complex step of 1e-7 (Surreal<double>), which agrees to
// O(1e-14) relative for these analytic functions. The identity "lambda" gives
// f = lambda and g = 1 exactly, as the reference does.
#pragma once

#include <cctype>
#include <cmath>
#include <cstdlib>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

namespace tmb {

struct Dual {
    double v = 0.0; // value
    double d = 0.0; // derivative with respect to lambda
    bool is_int = false;
};

class LambdaExpr {
  public:
    LambdaExpr() { parse("lambda"); }
    explicit LambdaExpr(const std::string &src) { parse(src); }

    const std::string &source() const { return src_; }
    bool is_identity() const { return identity_; }

    // f(lambda) and df/dlambda
    void eval(double lambda, double &f, double &g) const {
        if (identity_) {
            f = lambda;
            g = 1.0;
            return;
        }
        const Dual r = nodes_[root_].eval(*this, lambda);
        f = r.v;
        g = r.d;
    }

  private:
    enum class Op {
        Num, Lambda, Neg, Not, Add, Sub, Mul, Div, Mod, Lt, Le, Gt, Ge, Eq, Ne, And, Or, Cond, Call
    };
    struct Node {
        Op op = Op::Num;
        double num = 0.0;
        bool num_int = false;
        std::string fn;
        std::vector<int> kids;
        Dual eval(const LambdaExpr &e, double lambda) const { return e.eval_node(*this, lambda); }
    };

    std::string src_;
    bool identity_ = false;
    std::vector<Node> nodes_;
    int root_ = -1;
    size_t pos_ = 0;

    [[noreturn]] void fail(const std::string &why) const {
        throw std::invalid_argument("lambda transform \"" + src_ + "\": " + why + " at offset " + std::to_string(pos_));
    }

    void parse(const std::string &src) {
        src_ = src;
        nodes_.clear();
        pos_ = 0;
        root_ = parse_cond();
        skip();
        if (pos_ != src_.size()) {
            fail("unexpected character '" + std::string(1, src_[pos_]) + "'");
        }
        identity_ = nodes_[root_].op == Op::Lambda;
    }

    int add(Node n) {
        nodes_.push_back(std::move(n));
        return (int)nodes_.size() - 1;
    }
    int make(Op op, std::vector<int> kids) {
        Node n;
        n.op = op;
        n.kids = std::move(kids);
        return add(std::move(n));
    }

    void skip() {
        while (pos_ < src_.size() && std::isspace((unsigned char)src_[pos_])) {
            pos_++;
        }
    }
    bool accept(const char *tok) {
        skip();
        const size_t n = std::char_traits<char>::length(tok);
        if (src_.compare(pos_, n, tok) == 0) {
            // a one-character operator must not be the start of a longer one
            if (n == 1 && pos_ + 1 < src_.size()) {
                const char c = tok[0], next = src_[pos_ + 1];
                if ((c == '<' || c == '>' || c == '!' || c == '=') && next == '=') {
                    return false;
                }
                if ((c == '&' && next == '&') || (c == '|' && next == '|')) {
                    return false;
                }
            }
            pos_ += n;
            return true;
        }
        return false;
    }
    void expect(const char *tok) {
        if (!accept(tok)) {
            fail(std::string("expected '") + tok + "'");
        }
    }

    int parse_cond() {
        const int c = parse_or();
        if (accept("?")) {
            const int a = parse_cond();
            expect(":");
            const int b = parse_cond();
            return make(Op::Cond, {c, a, b});
        }
        return c;
    }
    int parse_or() {
        int l = parse_and();
        while (accept("||")) {
            l = make(Op::Or, {l, parse_and()});
        }
        return l;
    }
    int parse_and() {
        int l = parse_eq();
        while (accept("&&")) {
            l = make(Op::And, {l, parse_eq()});
        }
        return l;
    }
    int parse_eq() {
        int l = parse_rel();
        for (;;) {
            if (accept("==")) {
                l = make(Op::Eq, {l, parse_rel()});
            } else if (accept("!=")) {
                l = make(Op::Ne, {l, parse_rel()});
            } else {
                return l;
            }
        }
    }
    int parse_rel() {
        int l = parse_add();
        for (;;) {
            if (accept("<=")) {
                l = make(Op::Le, {l, parse_add()});
            } else if (accept(">=")) {
                l = make(Op::Ge, {l, parse_add()});
            } else if (accept("<")) {
                l = make(Op::Lt, {l, parse_add()});
            } else if (accept(">")) {
                l = make(Op::Gt, {l, parse_add()});
            } else {
                return l;
            }
        }
    }
    int parse_add() {
        int l = parse_mul();
        for (;;) {
            if (accept("+")) {
                l = make(Op::Add, {l, parse_mul()});
            } else if (accept("-")) {
                l = make(Op::Sub, {l, parse_mul()});
            } else {
                return l;
            }
        }
    }
    int parse_mul() {
        int l = parse_unary();
        for (;;) {
            if (accept("*")) {
                l = make(Op::Mul, {l, parse_unary()});
            } else if (accept("/")) {
                l = make(Op::Div, {l, parse_unary()});
            } else if (accept("%")) {
                l = make(Op::Mod, {l, parse_unary()});
            } else {
                return l;
            }
        }
    }
    int parse_unary() {
        if (accept("-")) {
            return make(Op::Neg, {parse_unary()});
        }
        if (accept("+")) {
            return parse_unary();
        }
        if (accept("!")) {
            return make(Op::Not, {parse_unary()});
        }
        return parse_primary();
    }
    int parse_primary() {
        skip();
        if (pos_ >= src_.size()) {
            fail("unexpected end of expression");
        }
        const char c = src_[pos_];
        if (c == '(') {
            pos_++;
            const int e = parse_cond();
            expect(")");
            return e;
        }
        if (std::isdigit((unsigned char)c) || c == '.') {
            return parse_number();
        }
        if (std::isalpha((unsigned char)c) || c == '_') {
            const size_t b = pos_;
            while (pos_ < src_.size() && (std::isalnum((unsigned char)src_[pos_]) || src_[pos_] == '_')) {
                pos_++;
            }
            const std::string id = src_.substr(b, pos_ - b);
            if (id == "lambda") {
                Node n;
                n.op = Op::Lambda;
                return add(n);
            }
            if (id == "PI") {
                // the reference's #define PI (k_lambda_transformer_jit.cuh:6), a double literal
                Node n;
                n.op = Op::Num;
                n.num = 3.141592653589793115997963468544185161;
                return add(n);
            }
            if (!accept("(")) {
                pos_ = b;
                fail("unknown identifier '" + id + "'");
            }
            Node n;
            n.op = Op::Call;
            n.fn = id;
            if (!accept(")")) {
                n.kids.push_back(parse_cond());
                while (accept(",")) {
                    n.kids.push_back(parse_cond());
                }
                expect(")");
            }
            const int arity = (id == "pow" || id == "atan2" || id == "fmin" || id == "fmax" || id == "min" ||
                               id == "max")
                                  ? 2
                                  : 1;
            static const char *known[] = {"sin",  "cos",  "tan",  "asin", "acos",  "atan",  "atan2", "sinh",
                                          "cosh", "tanh", "exp",  "log",  "log10", "sqrt",  "pow",   "fabs",
                                          "abs",  "fmin", "fmax", "min",  "max",   "floor", "ceil"};
            bool ok = false;
            for (const char *k : known) {
                ok = ok || id == k;
            }
            if (!ok) {
                fail("unknown function '" + id + "'");
            }
            if ((int)n.kids.size() != arity) {
                fail("function '" + id + "' takes " + std::to_string(arity) + " argument(s)");
            }
            return add(std::move(n));
        }
        fail("unexpected character '" + std::string(1, c) + "'");
    }
    int parse_number() {
        const char *start = src_.c_str() + pos_;
        char *end = nullptr;
        const double v = std::strtod(start, &end);
        if (end == start) {
            fail("bad number");
        }
        bool is_int = true;
        for (const char *p = start; p < end; p++) {
            if (*p == '.' || *p == 'e' || *p == 'E') {
                is_int = false;
            }
        }
        pos_ += (size_t)(end - start);
        // C suffixes: f / F (float literal: rounded to float), l / L, u / U
        if (pos_ < src_.size() && (src_[pos_] == 'f' || src_[pos_] == 'F') && !is_int) {
            pos_++;
            Node n;
            n.op = Op::Num;
            n.num = (double)(float)v;
            return add(n);
        }
        while (pos_ < src_.size() && (src_[pos_] == 'l' || src_[pos_] == 'L' || src_[pos_] == 'u' || src_[pos_] == 'U')) {
            pos_++;
        }
        Node n;
        n.op = Op::Num;
        n.num = v;
        n.num_int = is_int;
        return add(n);
    }

    static Dual num(double v, bool is_int = false) { return Dual{v, 0.0, is_int}; }
    static Dual truth(bool b) { return Dual{b ? 1.0 : 0.0, 0.0, true}; }

    Dual eval_node(const Node &n, double lambda) const {
        auto kid = [&](int k) { return nodes_[n.kids[k]].eval(*this, lambda); };
        switch (n.op) {
        case Op::Num:
            return num(n.num, n.num_int);
        case Op::Lambda:
            return Dual{lambda, 1.0, false};
        case Op::Neg: {
            const Dual a = kid(0);
            return Dual{-a.v, -a.d, a.is_int};
        }
        case Op::Not:
            return truth(kid(0).v == 0.0);
        case Op::Add: {
            const Dual a = kid(0), b = kid(1);
            return Dual{a.v + b.v, a.d + b.d, a.is_int && b.is_int};
        }
        case Op::Sub: {
            const Dual a = kid(0), b = kid(1);
            return Dual{a.v - b.v, a.d - b.d, a.is_int && b.is_int};
        }
        case Op::Mul: {
            const Dual a = kid(0), b = kid(1);
            return Dual{a.v * b.v, a.d * b.v + a.v * b.d, a.is_int && b.is_int};
        }
        case Op::Div: {
            const Dual a = kid(0), b = kid(1);
            if (a.is_int && b.is_int) {
                if (b.v == 0.0) {
                    throw std::invalid_argument("lambda transform \"" + src_ + "\": integer division by zero");
                }
                return num((double)((long long)a.v / (long long)b.v), true);
            }
            return Dual{a.v / b.v, (a.d * b.v - a.v * b.d) / (b.v * b.v), false};
        }
        case Op::Mod: {
            const Dual a = kid(0), b = kid(1);
            if (!(a.is_int && b.is_int) || b.v == 0.0) {
                throw std::invalid_argument("lambda transform \"" + src_ + "\": % needs nonzero integer operands");
            }
            return num((double)((long long)a.v % (long long)b.v), true);
        }
        case Op::Lt:
            return truth(kid(0).v < kid(1).v);
        case Op::Le:
            return truth(kid(0).v <= kid(1).v);
        case Op::Gt:
            return truth(kid(0).v > kid(1).v);
        case Op::Ge:
            return truth(kid(0).v >= kid(1).v);
        case Op::Eq:
            return truth(kid(0).v == kid(1).v);
        case Op::Ne:
            return truth(kid(0).v != kid(1).v);
        case Op::And:
            return truth(kid(0).v != 0.0 && kid(1).v != 0.0);
        case Op::Or:
            return truth(kid(0).v != 0.0 || kid(1).v != 0.0);
        case Op::Cond: {
            const Dual c = kid(0);
            return c.v != 0.0 ? kid(1) : kid(2);
        }
        case Op::Call:
            return call(n, lambda);
        }
        return num(0.0);
    }

    Dual call(const Node &n, double lambda) const {
        const std::string &f = n.fn;
        const Dual a = nodes_[n.kids[0]].eval(*this, lambda);
        const double x = a.v, dx = a.d;
        if (n.kids.size() == 2) {
            const Dual b = nodes_[n.kids[1]].eval(*this, lambda);
            const double y = b.v, dy = b.d;
            if (f == "pow") {
                const double v = std::pow(x, y);
                // d(x^y) = y x^(y-1) dx + x^y log(x) dy (the second term only where dy != 0)
                double d = (dx != 0.0) ? y * std::pow(x, y - 1.0) * dx : 0.0;
                if (dy != 0.0) {
                    d += v * std::log(x) * dy;
                }
                return Dual{v, d, false};
            }
            if (f == "atan2") {
                const double r2 = x * x + y * y;
                return Dual{std::atan2(x, y), (y * dx - x * dy) / r2, false};
            }
            const bool take_a = (f == "fmin" || f == "min") ? !(y < x) : !(x < y);
            return take_a ? Dual{x, dx, a.is_int && b.is_int} : Dual{y, dy, a.is_int && b.is_int};
        }
        if (f == "sin") {
            return Dual{std::sin(x), std::cos(x) * dx, false};
        }
        if (f == "cos") {
            return Dual{std::cos(x), -std::sin(x) * dx, false};
        }
        if (f == "tan") {
            const double t = std::tan(x);
            return Dual{t, (1.0 + t * t) * dx, false};
        }
        if (f == "asin") {
            return Dual{std::asin(x), dx / std::sqrt(1.0 - x * x), false};
        }
        if (f == "acos") {
            return Dual{std::acos(x), -dx / std::sqrt(1.0 - x * x), false};
        }
        if (f == "atan") {
            return Dual{std::atan(x), dx / (1.0 + x * x), false};
        }
        if (f == "sinh") {
            return Dual{std::sinh(x), std::cosh(x) * dx, false};
        }
        if (f == "cosh") {
            return Dual{std::cosh(x), std::sinh(x) * dx, false};
        }
        if (f == "tanh") {
            const double t = std::tanh(x);
            return Dual{t, (1.0 - t * t) * dx, false};
        }
        if (f == "exp") {
            const double e = std::exp(x);
            return Dual{e, e * dx, false};
        }
        if (f == "log") {
            return Dual{std::log(x), dx / x, false};
        }
        if (f == "log10") {
            return Dual{std::log10(x), dx / (x * std::log(10.0)), false};
        }
        if (f == "sqrt") {
            const double r = std::sqrt(x);
            return Dual{r, dx / (2.0 * r), false};
        }
        if (f == "fabs" || f == "abs") {
            return x < 0.0 ? Dual{-x, -dx, a.is_int} : Dual{x, dx, a.is_int};
        }
        if (f == "floor") {
            return Dual{std::floor(x), 0.0, false};
        }
        if (f == "ceil") {
            return Dual{std::ceil(x), 0.0, false};
        }
        throw std::invalid_argument("lambda transform \"" + src_ + "\": unknown function '" + f + "'");
    }
};

// The four schedules of one potential.
struct LambdaTransforms {
    LambdaExpr charge, sigma, epsilon, w;
    bool identity() const {
        return charge.is_identity() && sigma.is_identity() && epsilon.is_identity() && w.is_identity();
    }
};

} // namespace tmb
