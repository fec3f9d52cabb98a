"""Oracle (test infrastructure): CPU restatement and the reference build."""
