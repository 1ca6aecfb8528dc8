// Entry point of the oracle build: the reference's own main() is compiled as
// kapsel_main (-Dmain=kapsel_main) and called unchanged with the same argv.
int kapsel_main(int argc, char *argv[]);
int main(int argc, char *argv[]) { return kapsel_main(argc, argv); }
