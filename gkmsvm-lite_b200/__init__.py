"""B200-native gapped-k-mer SVM kernel path (package body filled in below)."""
