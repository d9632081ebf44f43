OPENQASM 2.0;
include "qelib1.inc";
gate majority a,b,c
{
cx c,b;
cx c,a;
ccx a,b,c;
}
gate unmaj a,b,c
{
ccx a,b,c;
cx c,a;
cx a,b;
}
gate adder a,b,c
{
majority a,b,c;
unmaj a,b,c;
}
qreg q[4];
creg c[4];
x q[0];
h q[3];
majority q[0],q[1],q[2];
rz(pi/4) q[3];
unmaj q[0],q[1],q[2];
adder q[3],q[2],q[1];
measure q[2] -> c[2];
