"""Host oracle (test infrastructure): a C++/OpenMP restatement of the
pyrochlore Monte Carlo used to check the engine. Only the tests, the smoke
check and the CPU-baseline leg of the benchmark import it."""
