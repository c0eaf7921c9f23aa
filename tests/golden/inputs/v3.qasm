OPENQASM 3;
include "stdgates.inc";
qubit[5] q;
bit[2] c;
h q[0:3];
cx q[0], q[1];
rz(-pi/4 + 2*0.1) q[2];
rzz(tau/8) q[2],q[3];
/* block */ cz q[3],q[4]; // tail
barrier q;
u(1e-1, .5, -2.5e0) q[4];
c[0] = measure q[0];
bit x = measure q[1];
