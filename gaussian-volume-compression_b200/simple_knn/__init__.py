"""Drop-in for the `simple_knn` extension imported by scene/gaussian_model.py:16."""
