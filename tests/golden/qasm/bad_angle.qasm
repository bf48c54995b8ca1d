OPENQASM 2.0;
qreg q[2];
h q[0];
rx(pi/2) q[1];
h q[1];
