"""OpenQASM test programs for the from_qasm / to_qasm parity tests.

Written for this project to exercise every construct ket's OpenQASM subset
accepts (bindings/qasm/qasm.cpp) and every error it reports.  make_golden.py
records what ket itself does with each one (tests/golden/qasm.json).
"""

HEADER = 'OPENQASM 2.0;\ninclude "qelib1.inc";\n'

# (name, source) -- programs ket accepts
PROGRAMS = [
    ("every_builtin", HEADER + """qreg q[4];
h q[0]; x q[1]; y q[2]; z q[3]; s q[0]; sdg q[1]; t q[2]; tdg q[3]; id q[0];
ch q[0],q[1]; cx q[1],q[2]; cy q[2],q[3]; cz q[3],q[0]; swap q[0],q[2];
ccx q[0],q[1],q[3]; cswap q[3],q[0],q[1];
rx(0.1) q[0]; ry(0.2) q[1]; rz(0.3) q[2];
crx(0.4) q[0],q[3]; cry(0.5) q[1],q[0]; crz(0.6) q[2],q[1];
cp(0.7) q[3],q[2]; cu1(0.8) q[0],q[1];
cu3(0.9,1.0,1.1) q[1],q[3]; cu(1.2,1.3,1.4) q[2],q[0];
U(1.5,1.6,1.7) q[3]; u(1.8,1.9,2.0) q[0]; u3(2.1,2.2,2.3) q[1];
u2(2.4,2.5) q[2]; u1(2.6) q[3]; p(2.7) q[0]; phase(2.8) q[1];
"""),
    ("angle_expressions", HEADER + """qreg q[2];
rz(pi) q[0]; rz(-pi/2) q[1]; rz(3*pi/4) q[0]; rz(-3*pi/7+1) q[1];
rx(.5) q[0]; rx(5.) q[1]; ry(1e-3) q[0]; ry(2.5E+1) q[1];
rz(--1) q[0]; rz(+-0.5) q[1]; rz( 2 * pi - 1 / -3 ) q[0];
rx(0x1p-2) q[1]; rx(0x.8) q[0]; ry(1 - 2 - 3) q[1]; ry(8/4/2) q[0];
u(pi/2, -pi, 2*pi/3) q[1]; cp(pi/12) q[0],q[1]; crz(-5*pi/6) q[1],q[0];
"""),
    ("registers_measure_barrier", HEADER + """qreg a[2];
qreg b[3];
creg x[2];
creg y[4];
h a[0]; cx a[0], b[2]; barrier a; barrier a[1], b[0]; barrier b, a[0];
measure a[0] -> y[3]; measure b[2] -> x[1]; measure b[0]->y[0];
"""),
    ("comments_and_spacing", """// leading line comment
OPENQASM 2.0; /* block
comment over lines */ include "qelib1.inc";
qreg   q [ 3 ] ;   creg c[3];
h  q[0] ;cx q[0] ,q[1];// trailing
  rz ( pi / 4 )   q [ 2 ] ;
/* x q[0]; */ y q[1];
t q[2]; /* unterminated to the end
z q[0];
"""),
    ("user_gates", HEADER + """gate bell a, b { h a; cx a, b; }
gate rot(theta, phi) t { rz(phi) t; ry(theta/2) t; rz(-phi) t; }
gate both(x) a, b { rot(x, x/3) a; bell a, b; rot(2*x, 0) b; }
gate noargs() a { s a; }
qreg q[4];
bell q[0], q[1];
rot(pi/3, 0.25) q[2];
both(0.7) q[3], q[0];
both(0.7) q[1], q[2];
both(1.1) q[2], q[3];
noargs() q[0];
"""),
    ("first_definition_wins", HEADER + """gate g a { x a; }
gate g a { y a; }
qreg q[2];
g q[0]; g q[1];
"""),
    ("gate_defs_before_or_after_use", HEADER + """qreg q[3];
late q[0], q[2];
gate late a, b { cz a, b; h b; }
late q[1], q[0];
"""),
    ("empty_and_zero_qubits", HEADER + """qreg q[0];
creg c[0];
"""),
    ("divide_by_zero_angle", HEADER + """qreg q[1];
rz(1/0) q[0]; rx(-1/0) q[0]; ry(0/0) q[0]; rz(1/-0) q[0];
"""),
    ("number_forms", HEADER + """qreg q[1];
rx(0x1.8p1) q[0]; rx(1.e5) q[0]; rz(0X.4P+3) q[0]; ry(007) q[0];
"""),
    ("builtins_shadow_user_gates", HEADER + """gate h a { x a; }
gate k(b) y { g(b+1) y; g(-b) y; }
gate g(a) x { rz(a*2) x; }
qreg q[2];
h q[0]; k(0.5) q[1]; k(0.5) q[0]; k(0.25) q[0];
"""),
    ("brick_wall_5q", HEADER + """qreg q[5];
U(0.11,0.22,0.33) q[0]; U(1.1,2.2,3.3) q[1]; U(0.5,0.6,0.7) q[2]; U(2.0,1.0,0.5) q[3]; U(0.9,0.8,0.7) q[4];
cx q[0],q[1]; cx q[2],q[3];
U(0.3,0.2,0.1) q[0]; U(1.3,1.2,1.1) q[1]; U(2.3,2.2,2.1) q[2]; U(0.4,0.4,0.4) q[3]; U(1.7,0.3,2.9) q[4];
cx q[1],q[2]; cx q[3],q[4];
"""),
]

# (name, source) -- programs ket rejects
ERRORS = [
    ("unsupported_gate", "qreg q[2]; foo q[0];"),
    ("uppercase_cx", "qreg q[2]; CX q[0],q[1];"),
    ("opaque", "qreg q[1]; opaque g a;"),
    ("if", "qreg q[1]; creg c[1]; if (c==1) x q[0];"),
    ("measure_without_arrow", "qreg q[1]; creg c[1]; measure q[0] c[0];"),
    ("unknown_register", "qreg q[1]; x r[0];"),
    ("index_out_of_range", "qreg q[2]; h q[2];"),
    ("negative_index", "qreg q[2]; h q[-1];"),
    ("angle_overflow", "qreg q[1]; rx(1e999) q[0];"),
    ("angle_underflow", "qreg q[1]; rx(1e-310) q[0];"),
    ("angle_dangling_exponent", "qreg q[1]; rx(1e+) q[0];"),
    ("angle_bare_hex_prefix", "qreg q[1]; rz(0x) q[0];"),
    ("unindexed_operand", "qreg q[2]; h q;"),
    ("malformed_declaration", "qreg q;"),
    ("wrong_qubit_count", "qreg q[3]; cx q[0];"),
    ("too_many_qubits", "qreg q[3]; h q[0], q[1];"),
    ("bad_angle_comma", "qreg q[1]; rx(1,2) q[0];"),
    ("bad_angle_suffix", "qreg q[1]; rz(2pi) q[0];"),
    ("bad_angle_symbol", "qreg q[1]; rz($) q[0];"),
    ("unknown_identifier", "qreg q[1]; rz(tau) q[0];"),
    ("missing_angle", "qreg q[1]; rx() q[0];"),
    ("missing_angle_no_parens", "qreg q[1]; rx q[0];"),
    ("missing_close_paren_statement", "qreg q[1]; rx(0.5 q[0];"),
    ("missing_close_paren_angle", "qreg q[1]; rx((0.5) q[0];"),
    # a parameter list ends at its first ')', so parentheses inside an angle
    # never parse in a gate statement
    ("nested_parentheses", "qreg q[1]; rz((1+2)*pi/7) q[0];"),
    ("u_two_angles", "qreg q[1]; U(1,2) q[0];"),
    ("u2_three_angles", "qreg q[1]; u2(1,2,3) q[0];"),
    ("u1_no_angle", "qreg q[1]; u1() q[0];"),
    ("cu3_two_angles", "qreg q[2]; cu3(1,2) q[0],q[1];"),
    ("gate_missing_name", "gate (a) x { h x; } qreg q[1];"),
    ("gate_missing_paren", "gate g(a x { h x; } qreg q[1];"),
    ("gate_missing_brace", "gate g a h a; qreg q[1];"),
    ("gate_no_qubits", "gate g(a) { h a; } qreg q[1];"),
    ("gate_param_count", "gate g(a) x { rz(a) x; } qreg q[1]; g(1,2) q[0];"),
    ("gate_qubit_count", "gate g x, y { cx x, y; } qreg q[2]; g q[0];"),
    ("gate_unknown_formal", "gate g x { h z; } qreg q[1]; g q[0];"),
    ("gate_body_barrier", "gate g x { barrier x; } qreg q[1]; g q[0];"),
    ("gate_unknown_param", "gate g(a) x { rz(b) x; } qreg q[1]; g(1) q[0];"),
    ("repeated_operand", "qreg q[2]; cx q[1], q[1];"),
    ("index_not_a_number", "qreg q[2]; h q[a];"),
]

# angles for the to_qasm formatting sweep (each as rz on a 1-qubit circuit)
ANGLES = [0.0, -0.0, 1e-13, -1e-13, 1e-11, 3.141592653589793, -3.141592653589793,
          1.5707963267948966, 2.0943951023931953, -2.356194490192345, 0.2617993877991494,
          0.28559933214452665, 0.4487989505128276, 11.0 * 3.141592653589793 / 12.0,
          13.0 * 3.141592653589793 / 12.0, 24.0 * 3.141592653589793, 1000.0 * 3.141592653589793 / 7.0,
          0.1, 1.0, 2.0, 0.123456789012345678, 1e-5, 123456.789, 1e20, -7.25,
          3.141592653589793 * (1.0 + 1e-10), 3.141592653589793 * (1.0 + 1e-8)]
