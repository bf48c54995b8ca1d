// mixed circuit: every gate the reader accepts, plus skipped commands
OPENQASM 2.0;
include "qelib1.inc";
qreg q[5];
creg c[5];
h q[0]; x q[1];
y q[2];
z q[3];
rx(0.25) q[4];
ry(1.5707963267948966) q[0];
rz(-0.7) q[1];
p(2.1) q[2];
cx q[0], q[1];
cy q[1],q[3];
cz q[4], q[0];
swap q[2], q[4];

   h   q[ 3 ] ;
barrier q[0],q[1];
s q[1];
measure q[0] -> c[0];
rx(3.0e-1) q[2];
