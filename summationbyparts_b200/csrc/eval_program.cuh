// Boundary data from expressions (BoundaryCharacteristic::Eval, euler/src/lib.rs:853-863): the
// multigrid driver's evalexpr expressions (multigrid/src/eval/evalexpr.rs) compiled on the host
// into small stack programs over f64 (every integer-typed or variable-free part is folded into a
// constant there), run here for each edge point of an SBP_BC_EVAL side at the stage time.
//
// A program is a stream of int32 words: an opcode, then its operand for EV_CONST (constant
// index), EV_VAR (EvalVar), EV_LOAD / EV_STORE (local slot), EV_FN1 / EV_FN2 (function id).
// sbp_system_set_eval validates every program (opcodes, operand ranges, stack depth at most
// kEvalStack and exactly one value at the end, locals below kEvalLocals) before it reaches the
// device, so the interpreter needs no checks of its own.
#pragma once

#include <cstdint>

namespace sbp {

constexpr int kEvalCode = 512;    // words per program
constexpr int kEvalConsts = 256;  // constants shared by the four programs
constexpr int kEvalStack = 32;
constexpr int kEvalLocals = 16;

enum EvalOp : int {
    EV_CONST = 1, EV_VAR, EV_LOAD, EV_STORE,
    EV_ADD, EV_SUB, EV_MUL, EV_DIV, EV_MOD, EV_POW, EV_NEG,
    EV_LT, EV_GT, EV_LE, EV_GE, EV_EQ, EV_NE, EV_AND, EV_OR, EV_NOT,
    EV_SELECT,  // c, a, b -> c != 0 ? a : b
    EV_FN1, EV_FN2,
    EV_OPS_END
};
enum EvalVar : int { EVV_X, EVV_Y, EVV_T, EVV_RHO, EVV_RHOU, EVV_RHOV, EVV_U, EVV_V, EVV_COUNT };
enum EvalFn1 : int {
    EF_SIN, EF_COS, EF_TAN, EF_ASIN, EF_ACOS, EF_ATAN, EF_SINH, EF_COSH, EF_TANH, EF_ASINH, EF_ACOSH, EF_ATANH,
    EF_EXP, EF_EXP2, EF_LN, EF_LOG2, EF_LOG10, EF_SQRT, EF_CBRT, EF_ABS, EF_FLOOR, EF_CEIL, EF_ROUND, EF1_COUNT
};
enum EvalFn2 : int { EF_POW, EF_HYPOT, EF_ATAN2, EF_MIN, EF_MAX, EF_LOGB, EF2_COUNT };
enum EvalForm : int { EVAL_CONSERVATION = 0, EVAL_PRESSURE = 1 };

// The four programs of one evaluator: conservation form rho, rhou, rhov, e; pressure form
// rho, u, v, p.
struct EvalDev {
    int form;
    int len[4];
    int code[4][kEvalCode];
    double consts[kEvalConsts];
};

#ifdef __CUDACC__
__device__ inline double eval_fn1(int f, double a) {
    switch (f) {
        case EF_SIN: return sin(a);
        case EF_COS: return cos(a);
        case EF_TAN: return tan(a);
        case EF_ASIN: return asin(a);
        case EF_ACOS: return acos(a);
        case EF_ATAN: return atan(a);
        case EF_SINH: return sinh(a);
        case EF_COSH: return cosh(a);
        case EF_TANH: return tanh(a);
        case EF_ASINH: return asinh(a);
        case EF_ACOSH: return acosh(a);
        case EF_ATANH: return atanh(a);
        case EF_EXP: return exp(a);
        case EF_EXP2: return exp2(a);
        case EF_LN: return log(a);
        case EF_LOG2: return log2(a);
        case EF_LOG10: return log10(a);
        case EF_SQRT: return sqrt(a);
        case EF_CBRT: return cbrt(a);
        case EF_ABS: return fabs(a);
        case EF_FLOOR: return floor(a);
        case EF_CEIL: return ceil(a);
        default: return a < 0.0 ? -floor(-a + 0.5) : floor(a + 0.5);  // halves away from zero
    }
}

__device__ inline double eval_fn2(int f, double a, double b) {
    switch (f) {
        case EF_POW: return pow(a, b);
        case EF_HYPOT: return hypot(a, b);
        case EF_ATAN2: return atan2(a, b);
        case EF_MIN: return fmin(a, b);
        case EF_MAX: return fmax(a, b);
        default: return log(a) / log(b);
    }
}

// One program over the variables vars[EVV_COUNT].
__device__ inline double eval_run(const int* __restrict__ code, int len, const double* __restrict__ consts,
                                  const double* vars) {
    double st[kEvalStack];
    double loc[kEvalLocals];
    int sp = 0;
    for (int pc = 0; pc < len;) {
        const int op = code[pc++];
        switch (op) {
            case EV_CONST: st[sp++] = consts[code[pc++]]; break;
            case EV_VAR: st[sp++] = vars[code[pc++]]; break;
            case EV_LOAD: st[sp++] = loc[code[pc++]]; break;
            case EV_STORE: loc[code[pc++]] = st[--sp]; break;
            case EV_NEG: st[sp - 1] = -st[sp - 1]; break;
            case EV_NOT: st[sp - 1] = st[sp - 1] != 0.0 ? 0.0 : 1.0; break;
            case EV_FN1: {
                const int f = code[pc++];
                st[sp - 1] = eval_fn1(f, st[sp - 1]);
                break;
            }
            case EV_FN2: {
                const int f = code[pc++];
                const double b = st[--sp];
                st[sp - 1] = eval_fn2(f, st[sp - 1], b);
                break;
            }
            case EV_SELECT: {
                const double b = st[--sp], a = st[--sp];
                st[sp - 1] = st[sp - 1] != 0.0 ? a : b;
                break;
            }
            default: {
                const double b = st[--sp], a = st[sp - 1];
                double r;
                switch (op) {
                    case EV_ADD: r = a + b; break;
                    case EV_SUB: r = a - b; break;
                    case EV_MUL: r = a * b; break;
                    case EV_DIV: r = a / b; break;
                    case EV_MOD: r = fmod(a, b); break;
                    case EV_POW: r = pow(a, b); break;
                    case EV_LT: r = a < b ? 1.0 : 0.0; break;
                    case EV_GT: r = a > b ? 1.0 : 0.0; break;
                    case EV_LE: r = a <= b ? 1.0 : 0.0; break;
                    case EV_GE: r = a >= b ? 1.0 : 0.0; break;
                    case EV_EQ: r = a == b ? 1.0 : 0.0; break;
                    case EV_NE: r = a != b ? 1.0 : 0.0; break;
                    case EV_AND: r = (a != 0.0 && b != 0.0) ? 1.0 : 0.0; break;
                    default: r = (a != 0.0 || b != 0.0) ? 1.0 : 0.0; break;  // EV_OR
                }
                st[sp - 1] = r;
                break;
            }
        }
    }
    return st[0];
}

// Conserved state z at (x, y, t) (euler/src/eval.rs:72-100 for the pressure form).
__device__ inline void eval_state(const EvalDev& E, double gamma, double t, double x, double y, double z[4]) {
    double v[EVV_COUNT] = {x, y, t, 0.0, 0.0, 0.0, 0.0, 0.0};
    const double rho = eval_run(E.code[0], E.len[0], E.consts, v);
    v[EVV_RHO] = rho;
    if (E.form == EVAL_CONSERVATION) {
        const double rhou = eval_run(E.code[1], E.len[1], E.consts, v);
        const double rhov = eval_run(E.code[2], E.len[2], E.consts, v);
        v[EVV_RHOU] = rhou;
        v[EVV_RHOV] = rhov;
        z[0] = rho;
        z[1] = rhou;
        z[2] = rhov;
        z[3] = eval_run(E.code[3], E.len[3], E.consts, v);
    } else {
        const double u = eval_run(E.code[1], E.len[1], E.consts, v);
        const double vv = eval_run(E.code[2], E.len[2], E.consts, v);
        v[EVV_U] = u;
        v[EVV_V] = vv;
        const double p = eval_run(E.code[3], E.len[3], E.consts, v);
        z[0] = rho;
        z[1] = u * rho;
        z[2] = vv * rho;
        z[3] = p / (gamma - 1.0) + rho * (u * u + vv * vv) / 2.0;
    }
}
#endif

// Host check of one program (see the file comment); returns an error text or nullptr.
inline const char* eval_check(const int* code, int len, int nconsts) {
    if (len < 1 || len > kEvalCode) return "program length out of range";
    int sp = 0;
    // Programs are straight-line (EV_SELECT evaluates both operands), so a slot written in
    // program order before every read of it is written before the read at run time.
    bool stored[kEvalLocals] = {};
    for (int pc = 0; pc < len;) {
        const int op = code[pc++];
        const bool has_arg = op == EV_CONST || op == EV_VAR || op == EV_LOAD || op == EV_STORE || op == EV_FN1 ||
                             op == EV_FN2;
        if (op < EV_CONST || op >= EV_OPS_END) return "unknown opcode";
        int arg = 0;
        if (has_arg) {
            if (pc >= len) return "missing operand";
            arg = code[pc++];
        }
        switch (op) {
            case EV_CONST:
                if (arg < 0 || arg >= nconsts) return "constant index out of range";
                ++sp;
                break;
            case EV_VAR:
                if (arg < 0 || arg >= EVV_COUNT) return "variable out of range";
                ++sp;
                break;
            case EV_LOAD:
                if (arg < 0 || arg >= kEvalLocals) return "local slot out of range";
                if (!stored[arg]) return "local slot read before it is written";
                ++sp;
                break;
            case EV_STORE:
                if (arg < 0 || arg >= kEvalLocals) return "local slot out of range";
                if (sp < 1) return "stack underflow";
                stored[arg] = true;
                --sp;
                break;
            case EV_NEG:
            case EV_NOT:
                if (sp < 1) return "stack underflow";
                break;
            case EV_FN1:
                if (arg < 0 || arg >= EF1_COUNT) return "function out of range";
                if (sp < 1) return "stack underflow";
                break;
            case EV_FN2:
                if (arg < 0 || arg >= EF2_COUNT) return "function out of range";
                if (sp < 2) return "stack underflow";
                --sp;
                break;
            case EV_SELECT:
                if (sp < 3) return "stack underflow";
                sp -= 2;
                break;
            default:
                if (sp < 2) return "stack underflow";
                --sp;
                break;
        }
        if (sp > kEvalStack) return "stack deeper than the interpreter's";
    }
    return sp == 1 ? nullptr : "program does not leave exactly one value";
}

}  // namespace sbp
